"""Share-file formats (orq_b200/io.py) against ORQ's own files: the
employees fixtures that ORQ's I/O test reads (tests/test_io.cpp:30-110),
written by the reference, copied by tests/golden/make_io_fixtures.py."""
import os

import numpy as np

from orq_b200 import io

D = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "io")


def paths(stem):
    return [os.path.join(D, f"{stem}_3pc_{p}.csv") for p in range(3)]


def plaintext():
    rows = [list(map(int, ln.split(","))) for ln in open(os.path.join(D, "employees.csv")).read().split()[1:]]
    emp, reg, age = (np.array(c, dtype=np.int64) for c in zip(*rows))
    return emp, reg, age


def test_vector_share_files_open_to_the_ages():
    _, _, age = plaintext()
    S = io.read_party_shares(paths("employees_age_secrets"), 32, 4)
    ages32 = np.zeros(32, dtype=np.int64)
    ages32[:len(age)] = age
    assert np.array_equal((S[0] ^ S[1] ^ S[2]).view(np.int32), ages32)
    T = io.read_party_shares(paths("employees_sorted_age_secrets"), 32, 4)
    assert np.array_equal((T[0] ^ T[1] ^ T[2]).view(np.int32), np.sort(ages32))


def test_table_share_files_open_to_the_table():
    emp, reg, age = plaintext()
    cols, nread = io.read_table_shares(paths("employees_secrets"), 32, 4)
    assert nread == 32 and set(cols) == {"[##V]", "[AGE]", "[EMPLOYEE_ID]", "[REGION]"}
    op = {k: (S[0] ^ S[1] ^ S[2]).view(np.int32) for k, S in cols.items()}
    keep = op["[##V]"] != 0
    assert keep.sum() == len(age)
    assert np.array_equal(op["[AGE]"][keep], age)
    assert np.array_equal(op["[EMPLOYEE_ID]"][keep], emp)
    assert np.array_equal(op["[REGION]"][keep], reg)


def test_share_files_round_trip_and_check_overlap(tmp_path):
    S = io.read_party_shares(paths("employees_age_secrets"), 32, 4)
    out = [str(tmp_path / f"v_{p}.csv") for p in range(3)]
    io.write_party_shares(S, out)
    assert open(out[0]).read() == open(paths("employees_age_secrets")[0]).read()
    assert np.array_equal(io.read_party_shares(out, 32, 4), S)
    cols, _ = io.read_table_shares(paths("employees_secrets"), 32, 4)
    tout = [str(tmp_path / f"t_{p}.csv") for p in range(3)]
    io.write_table_shares(cols, 32, tout)
    assert open(tout[1]).read() == open(paths("employees_secrets")[1]).read()
    back, _ = io.read_table_shares(tout, 32, 4)
    assert all(np.array_equal(back[k], cols[k]) for k in cols)
    # a party file that disagrees with its neighbour on their common share
    bad = open(out[1]).read().splitlines()
    a, b = bad[0].split(",")
    bad[0] = f"{int(a) ^ 1},{b}"
    open(out[1], "w").write("\n".join(bad) + "\n")
    try:
        io.read_party_shares(out, 32, 4)
        raise AssertionError("overlap mismatch not detected")
    except ValueError:
        pass


def test_reader_accepts_spaces_and_skips_a_header(tmp_path):
    p = [str(tmp_path / f"h_{k}.csv") for k in range(3)]
    for k in range(3):
        open(p[k], "w").write("s0 s1\n" + "\n".join(f"{k} {(k + 1) % 3}" for _ in range(4)) + "\n")
    S = io.read_party_shares(p, 4, 8)
    assert S[:, 0].tolist() == [0, 1, 2]
