"""Copies the two physics tables the hot path reads from a psphray checkout
into this directory, unchanged:

  test/atomic_rates_Hui.txt  -> atomic_rates_Hui.txt   (14-column rate table)
  src/kernel.akline          -> kernel.akline          (SPH column depths)

    python -m psphray_b200.data.import_tables /path/to/psphray

They are data in the reference's own formats (read by psg_rate_table_load()
and psg_kernel_table_load()); the column-depth table cannot be regenerated
bit for bit from the kernel formula, so it is carried as is.
"""
import os
import shutil
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
FILES = {"test/atomic_rates_Hui.txt": "atomic_rates_Hui.txt", "src/kernel.akline": "kernel.akline"}


def main(root: str) -> None:
    for src, dst in FILES.items():
        shutil.copyfile(os.path.join(root, src), os.path.join(HERE, dst))
        print(dst)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python -m psphray_b200.data.import_tables /path/to/psphray")
    main(sys.argv[1])
