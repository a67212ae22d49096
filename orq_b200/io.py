"""Share files: ORQ's CSV formats for secret shares and plaintext tables.

Vector shares (EVector::output and the EVector(size, file) constructor,
include/core/containers/e_vector.h:249-348): one file per party, one line per
element holding that party's replicated shares separated by commas (spaces are
accepted on input, and a line with anything but digits, '-' and spaces is
skipped). In 3PC party p holds (S[p], S[p+1]), so the three parties' files
together hold S0, S1, S2 and overlap pairwise; reading checks the overlap.

Tables (EncodedTable::inputCSVTableData, inputCSVTableSecretShares and
outputCSVTableSecretShares, include/core/containers/tabular/
encoded_table.h:396-590): a header line of column names — "[NAME]_r" for
replication r in share files, in the table's std::map column order — then one
line per row.

Values are the shares as signed decimals of the share type, as the
reference's streams write them. Everything here is host-side file handling;
shares move to and from the device through the runtime.
"""
from __future__ import annotations

import numpy as np

_NUMERIC = set("-0123456789 ")
_UNSIGNED = {1: np.uint8, 2: np.uint16, 4: np.uint32, 8: np.uint64}


def _wrap(values, width):
    """Python ints (any sign) to the width's unsigned two's-complement values."""
    mask = (1 << (8 * width)) - 1
    return np.array([v & mask for v in values], dtype=_UNSIGNED[width])


def _signed(a):
    return a.view({1: np.int8, 2: np.int16, 4: np.int32, 8: np.int64}[a.dtype.itemsize])


def read_party_file(path, n, width):
    """One party's vector share file: (2, rows) unsigned shares, rows <= n
    (the EVector(size, file) constructor stops after n lines)."""
    cols = ([], [])
    with open(path) as f:
        for line in f:
            if len(cols[0]) >= n:
                break
            line = line.strip().replace(",", " ")
            if not line or not set(line) <= _NUMERIC:
                continue
            a, b = line.split()[:2]
            cols[0].append(int(a))
            cols[1].append(int(b))
    return np.stack([_wrap(c, width) for c in cols]) if cols[0] else np.zeros((2, 0), _UNSIGNED[width])


def read_party_shares(paths, n, width):
    """The three parties' files of one vector: (3, n) distinct shares S0, S1,
    S2 (rows past the files' end are zero shares). Raises ValueError when
    party p's second share differs from party p+1's first."""
    per = [read_party_file(p, n, width) for p in paths]
    S = np.zeros((3, n), dtype=_UNSIGNED[width])
    for p in range(3):
        rows = per[p].shape[1]
        S[p, :rows] = per[p][0]
    for p in range(3):
        q = (p + 1) % 3
        rows = min(per[p].shape[1], per[q].shape[1])
        if not np.array_equal(per[p][1, :rows], per[q][0, :rows]):
            raise ValueError(f"share files of parties {p} and {q} disagree on S{q}")
    return S


def write_party_shares(S, paths):
    """EVector::output for the three parties: party p writes S[p], S[p+1]."""
    sv = _signed(np.asarray(S))
    for p, path in enumerate(paths):
        with open(path, "w") as f:
            for a, b in zip(sv[p].tolist(), sv[(p + 1) % 3].tolist()):
                f.write(f"{a},{b}\n")


def read_csv_table(path, names, rows):
    """inputCSVTableData's parse on the input party: {column: int64 values}
    for the columns in the header (each must be one of `names`), at most
    `rows` rows, and the number of rows read."""
    with open(path) as f:
        header = f.readline().strip().split(",")
        for h in header:
            if h not in names:
                raise ValueError(f"Column {h} not found in schema!")
        data = {h: np.zeros(rows, dtype=np.int64) for h in header}
        r = 0
        for line in f:
            if r >= rows:
                break
            if not line.strip():
                continue
            for h, tok in zip(header, line.strip().split(",")):
                data[h][r] = int(tok)
            r += 1
    return data, r


def read_table_shares(paths, rows, width):
    """inputCSVTableSecretShares for the three parties' files: ({column:
    (3, rows) distinct shares}, rows read). Header tokens are NAME_r (the
    last '_' splits the replication index)."""
    per = []
    nread = None
    for path in paths:
        with open(path) as f:
            header = f.readline().strip().split(",")
            mapping = []
            for tok in header:
                k = tok.rfind("_")
                mapping.append((tok[:k], int(tok[k + 1:])) if k >= 0 else (tok, 0))
            vals = {c: [[], []] for c, _ in mapping}
            r = 0
            for line in f:
                if r >= rows:
                    break
                if not line.strip():
                    continue
                for (c, rep), tok in zip(mapping, line.strip().split(",")):
                    vals[c][rep].append(int(tok))
                r += 1
        per.append(vals)
        nread = r if nread is None else min(nread, r)
    out = {}
    for c in per[0]:
        S = np.zeros((3, rows), dtype=_UNSIGNED[width])
        for p in range(3):
            a, b = per[p][c]
            S[p, :len(a)] = _wrap(a, width)
            q = (p + 1) % 3
            if b and per[q][c][0] and not np.array_equal(_wrap(b, width)[:nread],
                                                         _wrap(per[q][c][0], width)[:nread]):
                raise ValueError(f"column {c}: share files of parties {p} and {q} disagree")
        out[c] = S
    return out, nread


def write_table_shares(columns, rows, paths):
    """outputCSVTableSecretShares for the three parties: columns is
    {name: (3, rows) shares} in the table's column order."""
    names = list(columns)
    sv = {c: _signed(np.asarray(columns[c])) for c in names}
    for p, path in enumerate(paths):
        q = (p + 1) % 3
        with open(path, "w") as f:
            f.write(",".join(f"{c}_{r}" for c in names for r in (0, 1)) + "\n")
            for i in range(rows):
                f.write(",".join(f"{sv[c][s][i]}" for c in names for s in (p, q)) + "\n")
