"""k_pass_b_rg (the residue-grouped column pass, height 4096, 256-row pruned
transforms) emulated thread by thread in numpy (CPU only).

The emulation follows the kernel's index maps literally: which thread holds
which value in each phase, the shared-memory address of every store and load
(block buffer blk[c][m'][s] with row stride 17 and column stride CS, the
transposes inside each warp's final-phase ranges), and the row each output
lands in.  It checks that

* the column pass of one item equals the FFT definition: y = IFFT4096(I' conj(F))
  * 4096 with F = FFT4096 of the 256 non-zero rows;
* every shared-memory address stays inside the block buffer, and a warp's
  transpose rows stay inside the ranges that the same warp reads in the final
  phase (so no barrier is needed around the transposes);
* no two lanes of a half-warp touch the same 8-byte bank pair in any phase
  (addresses distinct modulo 16 float2), so each access is one wavefront per
  half-warp.
"""
import numpy as np

T, Y, RS = 256, 4096, 17
CS = 256 * RS + 4
AP = 260
NT = 1024
W16 = np.exp(-2j * np.pi * np.outer(np.arange(16), np.arange(16)) / 16)   # forward DFT16 matrix


def _dft16(v, sign):
    """v: (..., 16) -> 16-point DFT over the last axis, sign -1 forward, +1 inverse."""
    m = W16 if sign < 0 else W16.conj()
    return v @ m.T


def _w(e, n, sign):
    return np.exp(sign * 2j * np.pi * np.asarray(e, dtype=np.float64) / n)


def _residue_roles():
    tid = np.arange(NT)
    return tid >> 6, tid & 15, (tid >> 4) & 3, tid >> 5        # s, q, c, warp


def _srow(c, warp, rho):
    """float2 index of row rho of a thread's transpose block (the kernel's TM_RG_ROW)."""
    return (c & 1) * CS + 136 * warp + (rho >> 3) * (2 * CS) + (rho & 7) * RS


def _half_warp_conflict_free(addr):
    """addr: (NT,) float2 indices of one access; every half-warp's 16 distinct mod 16."""
    a = addr.reshape(NT // 16, 16) % 16
    return all(len(set(row)) == 16 for row in a)


def emulate_item(A, Ip):
    """A: (256, 4) rows of the item's 4 columns; Ip: (4096, 4) I' columns.
    Returns the (4096, 4) column-pass output and the shared-memory access log."""
    s, q, c, warp = _residue_roles()
    blk = np.full(4 * CS, np.nan, complex)
    log = []
    # forward: v[r] = A[q + 16 r][c] W4096^(-(q + 16 r) s), staging address c * AP + q + 16 r
    r = np.arange(16)
    n = q[:, None] + 16 * r[None, :]
    st_addr = c[:, None] * AP + n
    assert st_addr.max() < 4 * AP
    log.append(("staging", st_addr))
    v = A[n, c[:, None]] * _w(-(n * s[:, None]), Y, 1)
    v = _dft16(v, -1)
    v = v * _w(-(q[:, None] * r[None, :]), 256, 1)            # W256^(-q k1)
    # transpose 1: write row q column r, read row r column q
    wr = np.array([[_srow(c[t], warp[t], q[t]) + rr for rr in range(16)] for t in range(NT)])
    rd = np.array([[_srow(c[t], warp[t], rr) + q[t] for rr in range(16)] for t in range(NT)])
    blk[wr] = v
    v = blk[rd]
    log += [("transpose write", wr), ("transpose read", rd)]
    v = _dft16(v, -1)                                           # F[s + 16 q + 256 r]
    k = s[:, None] + 16 * q[:, None] + 256 * r[None, :]
    F = v
    v = Ip[k, c[:, None]] * np.conj(F)
    # inverse residue part
    v = _dft16(v, +1)
    v = v * _w(q[:, None] * r[None, :], 256, 1)
    blk[wr] = v
    v = blk[rd]
    v = _dft16(v, +1)
    v = v * _w(s[:, None] * (q[:, None] + 16 * r[None, :]), Y, 1)
    # block write blk[c][q + 16 r][s]
    bw = c[:, None] * CS + (q[:, None] + 16 * r[None, :]) * RS + s[:, None]
    blk[:] = np.nan
    blk[bw] = v
    log.append(("block write", bw))
    # final phase: thread (fc, fm) reads s = 0..15 of row fm
    tid = np.arange(NT)
    fc, fm = tid & 3, tid >> 2
    br = fc[:, None] * CS + fm[:, None] * RS + r[None, :]
    log.append(("final read", br))
    v = _dft16(blk[br], +1)
    out = np.full((Y, 4), np.nan, complex)
    out[fm[:, None] + 256 * r[None, :], fc[:, None]] = v
    return out, F, k, log, (wr, rd, br)


def test_column_pass_matches_fft_definition():
    rng = np.random.default_rng(7)
    A = rng.normal(size=(256, 4)) + 1j * rng.normal(size=(256, 4))
    Ip = rng.normal(size=(Y, 4)) + 1j * rng.normal(size=(Y, 4))
    out, F, k, _, _ = emulate_item(A, Ip)
    s, q, c, _ = _residue_roles()
    pad = np.zeros((Y, 4), complex)
    pad[:256] = A
    Fref = np.fft.fft(pad, axis=0)
    assert np.abs(F - Fref[k, c[:, None]]).max() < 1e-9 * np.abs(Fref).max()
    ref = np.fft.ifft(Ip * np.conj(Fref), axis=0) * Y
    assert not np.isnan(out).any()
    assert np.abs(out - ref).max() < 1e-9 * np.abs(ref).max()


def test_shared_memory_ranges_and_banks():
    rng = np.random.default_rng(8)
    A = rng.normal(size=(256, 4)) + 0j
    Ip = rng.normal(size=(Y, 4)) + 0j
    _, _, _, log, (wr, rd, br) = emulate_item(A, Ip)
    for name, addr in log:
        assert addr.min() >= 0 and addr.max() < (4 * AP if name == "staging" else 4 * CS), name
        for j in range(addr.shape[1]):
            assert _half_warp_conflict_free(addr[:, j]), (name, j)
    # the block write covers blk[c][m'][s] exactly once
    bw = dict(log)["block write"]
    assert len(np.unique(bw)) == bw.size == 4 * 256 * 16
    # each warp's transpose rows lie inside the ranges the same warp reads in the final phase,
    # and different half-warps' transposes never share an address
    warp = np.arange(NT) >> 5
    owner = {}
    for t in range(NT):
        for a_ in br[t]:
            owner[int(a_)] = warp[t]
    for t in range(NT):
        for a_ in np.concatenate([wr[t], rd[t]]):
            assert owner.get(int(a_)) == warp[t]
    half = np.arange(NT) >> 4
    seen = {}
    for t in range(NT):
        for a_ in wr[t]:
            assert seen.setdefault(int(a_), half[t]) == half[t]


def test_shared_memory_budget():
    exch = 8 * 4 * CS
    staging = 8 * 4 * AP
    twiddles = 8 * NT
    item_list = 4 * 2048
    assert exch + 3 * staging + twiddles + item_list + 64 <= 232448
    assert CS % 16 == 4 and RS % 2 == 1


def _col_schedule(ngroups, nb, b, nblk):
    """ColSchedule of tm_kernels.cuh: a block's (group, orientation) items in order."""
    rounds, rem = divmod(ngroups, nblk)
    parts = min(nb, nblk // rem) if rem else 1
    items = [(r * nblk + b, o) for r in range(rounds) for o in range(nb)]
    if rem and b < rem * parts:
        p = b // rem
        g = rounds * nblk + b % rem
        items += [(g, o) for o in range(p * nb // parts, (p + 1) * nb // parts)]
    return items


def test_column_schedule_covers_every_item_once():
    """Every (column group, orientation) item goes to exactly one block, blocks
    of one round hold adjacent groups at the same orientation step, and no block
    has more than a round's work beyond the average."""
    for ngroups, nb, nblk in [(513, 128, 148), (513, 32, 148), (513, 128, 296), (129, 256, 148), (5, 16, 148),
                              (1025, 64, 148), (17, 1, 148)]:
        lists = [_col_schedule(ngroups, nb, b, nblk) for b in range(nblk)]
        seen = [it for lst in lists for it in lst]
        assert len(seen) == len(set(seen)) == ngroups * nb
        longest = max(len(lst) for lst in lists)
        assert longest <= -(-ngroups // nblk) * nb
        # within the whole rounds, step i of every block is the same orientation on adjacent groups
        rounds = ngroups // nblk
        for i in range(0, rounds * nb, max(1, nb // 3)):
            step = sorted(lists[b][i] for b in range(nblk))
            assert {o for _, o in step} == {i % nb}
            gs = [g for g, _ in step]
            assert gs == list(range(gs[0], gs[0] + nblk))
