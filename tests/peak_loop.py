"""The reference's result-aggregation peak loop (match_template.cpp:1865-1928)
restated in numpy: the checker of the peak lists the host library and the
match_template program produce."""
import numpy as np


def reference_peaks(z, maps, threshold, radius, T, pixel_size):
    """The reference's peak loop (match_template.cpp:1865-1928) in numpy."""
    z = z.copy()
    ny, nx = z.shape
    e = T // 4 + 1
    out = []
    while len(out) < 1000:
        sub = z[e:ny - e + 1, e:nx - e + 1]
        k = int(np.argmax(sub))            # first maximum in scan order
        j, i = divmod(k, sub.shape[1])
        j, i = j + e, i + e
        if z[j, i] < threshold:
            break
        rec = [i * pixel_size, j * pixel_size] + [m[j, i] for m in maps] + [z[j, i]]
        for jj in range(max(j - radius, 0), min(j + radius, ny)):
            for ii in range(max(i - radius, 0), min(i + radius, nx)):
                if (ii - i) ** 2 + (jj - j) ** 2 <= radius * radius:
                    z[jj, ii] = -np.finfo(np.float32).max
        out.append(rec)
    return np.array(out, np.float32).reshape(-1, 8)
