"""Copies the reference's example observation tables into tests/golden/.

The reference ships examples/00_checkerboard_iso/src_rec_file_ph.csv and
src_rec_file_gr.csv (25 stations x 16 periods, each station pair once: 4800
rows).  They are the only real observation tables of the reference; the
event-builder test loads them through sa_srcrec_load.  Run in the container
that holds the reference checkout:
    python tests/golden/make_fixtures.py /path/to/reference
"""
import os
import shutil
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def main(ref_root):
    src = os.path.join(ref_root, "examples", "00_checkerboard_iso")
    for name in ("src_rec_file_ph.csv", "src_rec_file_gr.csv"):
        shutil.copyfile(os.path.join(src, name), os.path.join(HERE, name))
        print("copied", name)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
