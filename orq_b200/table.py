"""EncodedTable — ORQ's relational layer over the device runtime.

Mirror of orq::relational::EncodedTable (include/core/containers/tabular/
encoded_table.h) and its join (include/core/operators/join.h:32-233). Every
column is a shared vector on the GPU; the table logic (schema, padding,
concatenation, projection) is host bookkeeping, and every protocol step goes
through the C ABI in the reference's order, so the shares of every column
equal those of the reference run with the same keys (radix sort protocol).

Column names follow the reference's convention: a name containing "[" is a
boolean-shared column, anything else is arithmetic-shared. The schema is kept
in the reference's std::map order (byte order of the names), which decides the
order in which data columns are permuted and therefore the PRG consumption.
"""
from __future__ import annotations

import numpy as np

from . import (ASC, DESC, ASharedVector, BSharedVector, Direction, SortingProtocol, aggregate, aggregators,
               bitonic_sort, distinct as _distinct, multiplex, shuffle_columns, table_sort, _torch)

JOIN_ID = "[##TID]"
VALID = "[##V]"
UNIQ = "[##UNIQ]"
VALID_TEMP = "[##VALID_TEMP]"
RESERVED = (JOIN_ID, VALID, UNIQ)
_COPY_LIKE = (aggregators.copy, aggregators.valid)


def is_bshared(name: str) -> bool:
    """EncodedTable::isBShared (encoded_table.h:1669)."""
    return "[" in name


class EncodedTable:
    """orq::relational::EncodedTable<int64_t> (8-byte shares; `width` 4 gives
    EncodedTable<int32_t>)."""

    def __init__(self, rt, columns: dict | None = None, rows: int = 0, name: str = "",
                 protocol: int = SortingProtocol.DEFAULT, width: int = 8):
        self.rt = rt
        self.WIDTH = width
        self.tableName = name
        # SortingProtocol of this table's sorts (the reference fixes it with
        # DEFAULT_SORT_PROTO); tables derived from it inherit it
        self.protocol = protocol
        self.schema: dict = {}
        self.rows = rows
        for k, v in (columns or {}).items():
            self.schema[k] = v
        self.configure_valid()

    # ---- construction ----------------------------------------------------
    @classmethod
    def secret_share(cls, rt, columns, names, party: int = 0, name: str = "",
                     protocol: int = SortingProtocol.DEFAULT, width: int = 8):
        """secret_share(columns, schema) (encoded_table.h:1687-1707) + the
        EncodedTable(contents) constructor (encoded_table.h:252-265)."""
        assert len(columns) == len(names)
        cols = {}
        for data, nm in zip(columns, names):
            d = np.ascontiguousarray(np.asarray(data).astype(np.int32 if width == 4 else np.int64))
            cols[nm] = (rt.secret_share_b if is_bshared(nm) else rt.secret_share_a)(d, party)
        rows = len(columns[0]) if columns else 0
        return cls(rt, cols, rows, name, protocol, width)

    @classmethod
    def with_schema(cls, rt, names, rows: int, name: str = "", protocol: int = SortingProtocol.DEFAULT,
                    width: int = 8):
        """EncodedTable(name, schema, size): zero columns and every row valid."""
        t = cls(rt, {}, rows, name, protocol, width)
        for nm in names:
            t.add_column(nm)
        return t

    # ---- share files (orq_b200.io; encoded_table.h:382-590) -----------------
    def inputCSVTableData(self, path, party: int = 0):
        """inputCSVTableData (encoded_table.h:396-483): the input party reads a
        plaintext CSV (header of column names), the valid column becomes 1 for
        the rows read unless the file has it, and every column, in schema
        order, is secret-shared by that party."""
        from . import io

        names = self.getColumnNames()
        data, nread = io.read_csv_table(path, names, self.rows)
        if VALID not in data:
            v = np.zeros(self.rows, dtype=np.int64)
            v[:nread] = 1
            data[VALID] = v
        for k in names:
            d = data.get(k, np.zeros(self.rows, dtype=np.int64)).astype(self._sdtype())
            self.schema[k] = (self.rt.secret_share_b if is_bshared(k) else self.rt.secret_share_a)(d, party)

    def inputCSVTableSecretShares(self, paths):
        """inputCSVTableSecretShares (encoded_table.h:495-562) for the three
        parties' files; when the files have no valid column, the rows read are
        made valid by party 0 secret-sharing ones."""
        from . import io

        cols, nread = io.read_table_shares(paths, self.rows, self.WIDTH)
        for k, S in cols.items():
            assert k in self.schema, f"column '{k}' not found"
            self.schema[k] = type(self.schema[k])(self.rt, self.rt._to_dev(S.view(self._sdtype()), self.WIDTH))
        if VALID in self.schema and VALID not in cols:
            ones = self.rt.secret_share_b(np.ones(nread, dtype=self._sdtype()), 0)
            self.schema[VALID].shares[:, :nread] = ones.shares

    def outputCSVTableSecretShares(self, paths):
        """outputCSVTableSecretShares (encoded_table.h:564-606): every column
        in schema order, header NAME_r, one file per party."""
        from . import io

        io.write_table_shares({k: self.schema[k].shares.cpu().numpy() for k in self.getColumnNames()},
                              self.rows, paths)

    def inputSecretShares(self, column, paths):
        """inputSecretShares (encoded_table.h:382-388): a column from vector
        share files."""
        v = self.rt.input_secret_shares(paths, self.rows, self.WIDTH, not is_bshared(column))
        self.schema[column] = v

    def outputSecretShares(self, column, paths):
        """outputSecretShares (encoded_table.h:608-620)."""
        self.schema[column].outputSecretShares(paths)

    def _sdtype(self):
        return np.int32 if self.WIDTH == 4 else np.int64

    def _zeros(self, name, n):
        t = self.rt._alloc(n, self.WIDTH)
        t.zero_()
        return (BSharedVector if is_bshared(name) else ASharedVector)(self.rt, t)

    def _ones(self, name, n):
        """public_share of 1: S0 = 1, S1 = S2 = 0."""
        v = self._zeros(name, n)
        v.shares[0].fill_(1)
        return v

    def configure_valid(self):
        """configureValid (encoded_table.h:272-284): all rows valid."""
        if VALID not in self.schema:
            self.add_column(VALID)
        self.schema[VALID] = self._ones(VALID, self.rows)

    # ---- schema ------------------------------------------------------------
    def size(self) -> int:
        return self.rows

    def getColumnNames(self):
        return sorted(self.schema)

    def __getitem__(self, name):
        return self.schema[name]

    def __setitem__(self, name, value):
        assert name in self.schema, f"column '{name}' not found"
        assert value.size() == self.rows
        self.schema[name] = value

    def add_column(self, name, rows: int | None = None):
        if name in self.schema:
            raise ValueError(f"Table column with name {name} already exists.")
        self.schema[name] = self._zeros(name, self.rows if rows is None else rows)

    def addColumns(self, names, rows: int | None = None):
        for nm in names:
            self.add_column(nm, rows)

    def deleteColumns(self, names):
        for nm in names:
            self.schema.pop(nm, None)

    def project(self, cols):
        """project (encoded_table.h:792-805): keep cols plus reserved columns."""
        keep = set(cols) | set(RESERVED)
        self.deleteColumns([k for k in self.getColumnNames() if k not in keep])

    def resize(self, n: int):
        """resize (encoded_table.h:1426-1436): truncate, or extend with zero rows."""
        if n == self.rows:
            return
        for k in self.getColumnNames():
            v = self.schema[k]
            new = self._zeros(k, n)
            m = min(n, self.rows)
            new.shares[:, :m] = v.shares[:, :m]
            self.schema[k] = new
        self.rows = n

    def head(self, n: int):
        self.resize(n)

    def tail(self, n: int):
        for k in self.getColumnNames():
            v = self.schema[k]
            self.schema[k] = type(v)(self.rt, v.shares[:, self.rows - n:].contiguous())
        self.rows = n

    def pad_power_of_two(self):
        """pad_power_of_two (encoded_table.h:1446-1468) with zero padding."""
        old = self.rows
        self.resize(1 << max(0, (old - 1).bit_length()) if old > 0 else 1)

    def filter(self, col):
        """filter (encoded_table.h:299-301): valid &= col."""
        self.schema[VALID] &= col

    # ---- concatenate (encoded_table.h:1548-1610) --------------------------
    def concatenate(self, other: "EncodedTable") -> "EncodedTable":
        new_schema = [JOIN_ID] + [c for c in self.getColumnNames() if c != JOIN_ID]
        new_schema += [c for c in other.getColumnNames() if c not in self.schema]
        n = self.rows + other.rows
        t = EncodedTable(self.rt, {}, n, self.tableName + "+" + other.tableName, self.protocol, self.WIDTH)
        for c in new_schema:
            if c not in t.schema:
                t.add_column(c)
        for c in self.getColumnNames():
            t.schema[c].shares[:, :self.rows] = self.schema[c].shares
        for c in other.getColumnNames():
            t.schema[c].shares[:, self.rows:n] = other.schema[c].shares
        # table id 1 for the other table's rows: one secret-shared 1, repeated
        one = self.rt.secret_share_b(np.ones(1, dtype=self._sdtype()), 0)
        t.schema[JOIN_ID].shares[:, self.rows:n] = one.shares[:, :1]
        return t

    # ---- sort (encoded_table.h:900-998) ------------------------------------
    def sort(self, columns, order=ASC, protocol=None):
        """Sorts the table on `columns` (names, or (name, order) pairs) with
        the quicksort or radix protocol (table_sort), or with the bitonic
        network on the table padded to a power of two (padding rows are cut
        again when the sort is on the valid column)."""
        spec = [(c, order) for c in columns] if not (columns and isinstance(columns[0], tuple)) else columns
        protocol = self.protocol if protocol is None else protocol
        original = self.rows
        if protocol == SortingProtocol.BITONICSORT:
            self.pad_power_of_two()
        keys = [c for c, _ in spec]
        orders = [o for _, o in spec]
        single_bit = [c in (VALID, JOIN_ID) for c in keys]
        can_unpad = VALID in keys
        unpad_from_top = dict(spec).get(VALID, ASC) == ASC
        data_a, data_b = [], []
        for k in self.getColumnNames():
            if k in keys:
                continue
            (data_b if is_bshared(k) else data_a).append(self.schema[k])
        key_cols = [self.schema[k] for k in keys]
        if protocol == SortingProtocol.BITONICSORT:
            bitonic_sort(key_cols, data_a, data_b, orders)
            if can_unpad:
                if unpad_from_top:
                    self.tail(original)
                else:
                    self.resize(original)
        else:
            table_sort(key_cols, data_a, data_b, orders, single_bit, protocol)
        return self

    # ---- shuffle, mask, finalize (encoded_table.h:170-222,645-652,1003-1018) -
    def shuffle(self):
        """EncodedTable::shuffle: every column (arithmetic ones first, then
        boolean, each in schema order) permuted by one secret permutation."""
        data_a, data_b = [], []
        for k in self.getColumnNames():
            (data_b if is_bshared(k) else data_a).append(self.schema[k])
        shuffle_columns(data_a, data_b)
        return self

    def mask(self, mask_column=VALID, keys=None):
        """EncodedTable::mask: rows whose mask bit is 0 get MASK_VALUE (the
        share type's maximum) in every other column, via multiplex on the
        bit (and on its b2a_bit for arithmetic columns); MASK_VALUE is
        secret-shared once by party 0, arithmetic sharing first."""
        sel_b = self.schema[mask_column]
        n = sel_b.size()
        sel_a = sel_b.b2a_bit()
        mv = np.array([(1 << (8 * self.WIDTH - 1)) - 1], dtype=self._sdtype())
        one_a = self.rt.secret_share_a(mv, 0)
        one_b = self.rt.secret_share_b(mv, 0)
        full_a = ASharedVector(self.rt, one_a.shares.expand(3, n).contiguous())
        full_b = BSharedVector(self.rt, one_b.shares.expand(3, n).contiguous())
        for k in (keys if keys is not None else self.getColumnNames()):
            if k == mask_column:
                continue
            c = self.schema[k]
            self.schema[k] = multiplex(sel_b, full_b, c) if is_bshared(k) else multiplex(sel_a, full_a, c)
        return self

    def finalize(self, do_shuffle=True):
        """EncodedTable::finalize: shuffle (optionally), then mask."""
        if do_shuffle:
            self.shuffle()
        return self.mask()

    # ---- distinct (encoded_table.h:1198-1212) -----------------------------
    def distinct_into(self, keys, res):
        r = _distinct([self.schema[k] for k in keys])
        self.schema[res] = r
        return self

    # ---- aggregate (encoded_table.h:1059-1186) -----------------------------
    def aggregate(self, keys, agg_spec, reverse=False, do_sort=True, mark_valid=True, table_id=None):
        keys = list(keys)
        if do_sort:
            keys = [VALID] + keys
            self.sort(keys, ASC)
        original = self.rows
        self.pad_power_of_two()
        keys_vec = [self.schema[k] for k in keys]
        b_agg, a_agg = [], []
        has_agg = False
        for data, result, func in agg_spec:
            assert is_bshared(data) == is_bshared(result)
            if func not in _COPY_LIKE:
                has_agg = True
            (b_agg if is_bshared(data) else a_agg).append((self.schema[data], self.schema[result], func))
        sel = None
        if mark_valid:
            self.addColumns([UNIQ])
            self.distinct_into(keys, UNIQ)
            if table_id is not None:
                sel = self.schema[table_id]
        aggregate(keys_vec, b_agg, a_agg, Direction.Reverse if reverse else Direction.Forward, sel)
        if original < self.rows:
            self.resize(original)
        if mark_valid:
            if has_agg:
                uniq = self.schema[UNIQ]
                if reverse:
                    # bottom row of each group stays valid
                    v = self.schema[VALID]
                    n = self.rows
                    head = BSharedVector(self.rt, v.shares[:, :n - 1].contiguous())
                    head &= BSharedVector(self.rt, uniq.shares[:, 1:].contiguous())
                    v.shares[:, :n - 1] = head.shares
                else:
                    self.filter(uniq)
            self.deleteColumns([UNIQ])
        return self

    # ---- join (join.h:32-233) ----------------------------------------------
    def _join(self, right, keys, agg_spec, left_outer=False, right_outer=False, anti=False,
              trim_invalid=True):
        concat = self.concatenate(right)
        out_cols = set(keys) | set(right.getColumnNames())
        for data, result, _ in agg_spec:
            out_cols.update((data, result))
        if left_outer:
            out_cols.update(self.getColumnNames())
        concat.project(sorted(out_cols))
        keys = [VALID] + list(keys)
        concat.sort(keys + [JOIN_ID])
        concat.addColumns([UNIQ, VALID_TEMP])
        agg_spec = list(agg_spec)
        if not right_outer:
            agg_spec.append((VALID_TEMP, VALID_TEMP, aggregators.valid))
            concat.distinct_into(keys, UNIQ)
        valid = concat.schema[VALID]
        if left_outer:
            if right_outer:
                concat.schema[VALID_TEMP] = BSharedVector(self.rt, valid.shares.clone())
            else:
                tid, uniq = concat.schema[JOIN_ID], concat.schema[UNIQ]
                concat.schema[VALID_TEMP] = valid & ~(tid & uniq)
                n = concat.rows
                vt = concat.schema[VALID_TEMP]
                head = BSharedVector(self.rt, vt.shares[:, :n - 1].contiguous())
                t = BSharedVector(self.rt, tid.shares[:, :n - 1].contiguous())
                u = BSharedVector(self.rt, uniq.shares[:, 1:].contiguous())
                head &= (t | u)
                vt.shares[:, :n - 1] = head.shares
        else:
            if right_outer:
                concat.schema[VALID_TEMP] = valid & concat.schema[JOIN_ID]
            else:
                concat.schema[VALID_TEMP] = valid & ~concat.schema[UNIQ]
        if anti:
            agg_spec.append((VALID_TEMP, VALID_TEMP, aggregators.copy))
        concat.deleteColumns([UNIQ])
        concat.aggregate(keys, agg_spec, reverse=True, do_sort=False, table_id=JOIN_ID)
        concat.filter(concat.schema[VALID_TEMP])
        concat.deleteColumns([VALID_TEMP, JOIN_ID])
        if trim_invalid and not left_outer:
            L, R = self.rows, right.rows
            w = 8 * self.WIDTH
            c = len(self.schema) - 1
            if R < (L * (w + c - 1)) // (c + 2):
                concat.sort([VALID], DESC)
                concat.head(R)
        return concat

    def inner_join(self, right, keys, agg_spec=(), trim_invalid=True):
        """EncodedTable::inner_join (join.h:235-243)."""
        return self._join(right, keys, agg_spec, trim_invalid=trim_invalid)

    def left_outer_join(self, right, keys, agg_spec=(), trim_invalid=True):
        return self._join(right, keys, agg_spec, left_outer=True, trim_invalid=trim_invalid)

    def right_outer_join(self, right, keys, agg_spec=(), trim_invalid=True):
        return self._join(right, keys, agg_spec, right_outer=True, trim_invalid=trim_invalid)

    def full_outer_join(self, right, keys, agg_spec=(), trim_invalid=True):
        return self._join(right, keys, agg_spec, left_outer=True, right_outer=True,
                          trim_invalid=trim_invalid)

    # ---- output ------------------------------------------------------------
    def open_with_schema(self, remove_invalid=True):
        """open_with_schema (encoded_table.h:672-711): opened columns in schema
        order, invalid rows removed."""
        data, names = [], []
        valid = None
        for k in self.getColumnNames():
            o = self.schema[k].open().cpu().numpy()
            if remove_invalid and k == VALID:
                valid = o
            else:
                data.append(o)
                names.append(k)
        if remove_invalid and valid is not None:
            keep = valid != 0
            data = [d[keep] for d in data]
        return data, names
