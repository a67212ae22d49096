"""Copy ORQ's share-file fixtures into tests/golden/io/.

The reference's I/O test (tests/test_io.cpp:30-110) reads secret shares that
ORQ itself wrote for a 32-row employees table (per-party CSV files of a
3-party replicated sharing) and its plaintext CSV. They pin the readers in
orq_b200/io.py: opening the shares must give the plaintext. The files are
reference-written data, copied unchanged.

Usage: python tests/golden/make_io_fixtures.py   (needs the reference tree; run
in the build container, not at test time)
"""
import os
import shutil

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(os.environ.get("ORQ_REF", "/root/reference"), "tests", "data")
FILES = ["employees.csv"] + [f"employees{s}_secrets_3pc_{p}.csv" for s in ("", "_age", "_sorted_age")
                             for p in range(3)]


def main():
    out = os.path.join(HERE, "io")
    os.makedirs(out, exist_ok=True)
    for f in FILES:
        shutil.copyfile(os.path.join(SRC, f), os.path.join(out, f))
        print(f)


if __name__ == "__main__":
    main()
