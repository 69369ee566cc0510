"""Regenerate the MRC fixtures of the reference's unit tests.

The reference's console_test program embeds three MRC files as byte arrays
(src/programs/console_test/hiv_image_80x80x1.cpp,
hiv_images_shift_noise_80x80x10.cpp, sine_128x128x1.cpp) and writes them to a
temporary directory before testing (console_test.cpp:1086-1107).  This script
parses those arrays out of the reference sources and writes the same bytes to
tests/golden/*.mrc.  It needs the reference tree, so it runs only where the
reference is mounted; the .mrc outputs are committed.

Usage: python tests/golden/make_console_fixtures.py <path of the cisTEM source tree>
"""
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
FILES = {
    "hiv_image_80x80x1.mrc": "hiv_image_80x80x1.cpp",
    "hiv_images_shift_noise_80x80x10.mrc": "hiv_images_shift_noise_80x80x10.cpp",
    "sine_wave_128x128x1.mrc": "sine_128x128x1.cpp",
}


def main():
    if len(sys.argv) != 2:
        sys.exit("usage: make_console_fixtures.py <path of the cisTEM source tree>")
    ref = sys.argv[1]
    src_dir = os.path.join(ref, "src", "programs", "console_test")
    for out_name, src_name in FILES.items():
        text = open(os.path.join(src_dir, src_name)).read()
        body = text[text.index("{") + 1: text.rindex("}")]
        data = bytes(int(h, 16) for h in re.findall(r"0x([0-9a-fA-F]{2})", body))
        with open(os.path.join(HERE, out_name), "wb") as f:
            f.write(data)
        print(f"{out_name}: {len(data)} bytes")


if __name__ == "__main__":
    main()
