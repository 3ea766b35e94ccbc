"""Result export to SQLite in the reference's row discipline: FixedSizeSQLDB
(src/hyteg/dataexport/SQL.hpp:33-130, SQL.cpp:24-57).

Constant entries go into every row and are fixed at the first write; variable entries must all be
set before each write (no empty cells); a value is set once per row unless overwriting is allowed.
Rows are stored through the storage scheme of waLBerla's sqlite module (the `walberla` submodule of
the reference, absent from its tree here, restated from its published behaviour): one table `runs`
with an integer key `runId` and a `timestamp`, and one column per entry, typed INTEGER, DOUBLE or
TEXT and added when first used. Host-only; no device work.
"""
import sqlite3

__all__ = ["FixedSizeSQLDB"]


def _kind(value):
    if isinstance(value, bool):
        return "i", int(value)
    if isinstance(value, int):
        return "i", int(value)
    if isinstance(value, float):
        return "d", float(value)
    if isinstance(value, str):
        return "s", value
    raise TypeError("SQL entry must be int, bool, float or str, not %s" % type(value).__name__)


class FixedSizeSQLDB:
    _SQL_TYPE = {"i": "INTEGER", "d": "DOUBLE", "s": "TEXT"}

    def __init__(self, dbFile, allowOverwritingValues=False):
        self.db_file = str(dbFile)
        self.allow_overwriting = bool(allowOverwritingValues)
        self.columns_fixed = False
        self.constant = {"i": {}, "d": {}, "s": {}}
        self.variable = {"i": {}, "d": {}, "s": {}}
        self.variable_keys = []
        with sqlite3.connect(self.db_file) as con:
            con.execute("CREATE TABLE IF NOT EXISTS runs (runId INTEGER PRIMARY KEY, "
                        "timestamp DATETIME DEFAULT CURRENT_TIMESTAMP)")

    def setConstantEntry(self, key, value):
        if self.columns_fixed:
            raise RuntimeError('Cannot insert "%s" since columns are fixed after first write.' % key)
        k, v = _kind(value)
        m = self.constant[k]
        if not self.allow_overwriting and key in m:
            raise RuntimeError('Attempt to overwrite "%s" dismissed.' % key)
        m[key] = v

    def setVariableEntry(self, key, value):
        if self.columns_fixed:
            if key not in self.variable_keys:
                raise RuntimeError('New variable key "%s" cannot be inserted since columns are fixed.' % key)
        elif key not in self.variable_keys:
            self.variable_keys.append(key)
        k, v = _kind(value)
        m = self.variable[k]
        if not self.allow_overwriting and key in m:
            raise RuntimeError('Attempt to overwrite "%s" dismissed.' % key)
        m[key] = v

    def writeRowOnRoot(self):
        """Stores the current row; every variable key must be set (exactly once across types)."""
        for key in self.variable_keys:
            if sum(key in self.variable[k] for k in "ids") != 1:
                raise RuntimeError('Variable key "%s" not set for this row.' % key)
        row = {}
        for k in "ids":
            for key, v in list(self.constant[k].items()) + list(self.variable[k].items()):
                row[key] = (k, v)
        with sqlite3.connect(self.db_file) as con:
            have = {r[1] for r in con.execute("PRAGMA table_info(runs)")}
            for key, (k, _) in row.items():
                if key not in have:
                    con.execute('ALTER TABLE runs ADD COLUMN "%s" %s' % (key.replace('"', '""'), self._SQL_TYPE[k]))
            keys = list(row)
            cols = ", ".join('"%s"' % c.replace('"', '""') for c in keys)
            con.execute("INSERT INTO runs (%s) VALUES (%s)" % (cols, ", ".join("?" * len(keys))),
                        [row[c][1] for c in keys])
        self.columns_fixed = True
        for k in "ids":
            self.variable[k].clear()
