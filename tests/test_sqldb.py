"""FixedSizeSQLDB (SQL.hpp:33-130, SQL.cpp:24-57) row discipline on a temporary SQLite file."""
import sqlite3

import pytest

from hyteg_b200.sqldb import FixedSizeSQLDB


def rows(path):
    con = sqlite3.connect(str(path))
    con.row_factory = sqlite3.Row
    out = [dict(r) for r in con.execute("SELECT * FROM runs ORDER BY runId")]
    types = {r[1]: r[2] for r in con.execute("PRAGMA table_info(runs)")}
    con.close()
    return out, types


def test_rows_and_types(tmp_path):
    db = FixedSizeSQLDB(tmp_path / "r.db")
    db.setConstantEntry("level", 8)
    db.setConstantEntry("mesh", "cube_48el")
    db.setConstantEntry("omega", 1.0)
    for cycle, res in enumerate([1.0, 0.1, 0.01]):
        db.setVariableEntry("cycle", cycle)
        db.setVariableEntry("residual", res)
        db.writeRowOnRoot()
    out, types = rows(tmp_path / "r.db")
    assert [(r["cycle"], r["residual"], r["level"], r["mesh"], r["omega"]) for r in out] == [
        (0, 1.0, 8, "cube_48el", 1.0), (1, 0.1, 8, "cube_48el", 1.0), (2, 0.01, 8, "cube_48el", 1.0)]
    assert types["level"] == "INTEGER" and types["residual"] == "DOUBLE" and types["mesh"] == "TEXT"
    assert all(r["runId"] is not None and r["timestamp"] for r in out)


def test_discipline(tmp_path):
    db = FixedSizeSQLDB(tmp_path / "d.db")
    db.setConstantEntry("a", 1)
    with pytest.raises(RuntimeError, match="overwrite"):
        db.setConstantEntry("a", 2)
    db.setVariableEntry("x", 1.5)
    with pytest.raises(RuntimeError, match="overwrite"):
        db.setVariableEntry("x", 2.5)
    db.writeRowOnRoot()
    with pytest.raises(RuntimeError, match="not set for this row"):
        db.writeRowOnRoot()  # x missing
    with pytest.raises(RuntimeError, match="fixed"):
        db.setConstantEntry("b", 1)
    with pytest.raises(RuntimeError, match="cannot be inserted"):
        db.setVariableEntry("y", 1)
    db.setVariableEntry("x", 3.5)
    db.writeRowOnRoot()
    out, _ = rows(tmp_path / "d.db")
    assert [r["x"] for r in out] == [1.5, 3.5]


def test_overwriting_allowed_and_bools(tmp_path):
    db = FixedSizeSQLDB(tmp_path / "o.db", allowOverwritingValues=True)
    db.setConstantEntry("flag", True)
    db.setConstantEntry("flag", False)
    db.setVariableEntry("v", 1)
    db.setVariableEntry("v", 2)
    db.writeRowOnRoot()
    out, types = rows(tmp_path / "o.db")
    assert out[0]["flag"] == 0 and out[0]["v"] == 2 and types["flag"] == "INTEGER"
    with pytest.raises(TypeError):
        db.setVariableEntry("v", [1])
