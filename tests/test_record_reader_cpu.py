"""Records written by this repository's command-line drop-ins (ice_generate_phase,
rainbow_generate; tests/golden/records/, made on a GPU by tests/golden/make_record_fixtures.py)
opened by the reference's own record reader, PhaseRecord(validate=True) from
python/rainbow_dataset/record.py:19-158, unchanged -- the consumer contract of the reference's
datasets.  Without the reference checkout the restated contract in record_check.py stands in."""
from __future__ import annotations

import json
import shutil

import numpy as np
import pytest

from conftest import GOLDEN
from record_check import reference_reader, validate_record

RECORDS = sorted(p for p in (GOLDEN / "records").iterdir() if p.is_dir()) if (GOLDEN / "records").is_dir() else []


def test_fixture_records_exist():
    assert len(RECORDS) >= 3, "run tests/golden/make_record_fixtures.py on a GPU host"


@pytest.mark.parametrize("path", RECORDS, ids=[p.name for p in RECORDS])
def test_record_accepted(path):
    rec = validate_record(path)  # the reference reader too, where its checkout is present
    m = json.loads((path / "metadata.json").read_text())
    assert rec["phi"].shape == (m["phi_count"] + 1,)
    assert abs(rec["cell_probability"].sum() - 1) <= 1e-12


@pytest.mark.parametrize("path", RECORDS, ids=[p.name for p in RECORDS])
def test_reference_reader_accepts_record(path):
    reader = reference_reader()
    if reader is None:
        pytest.skip("reference checkout not present")
    rec = reader(path, validate=True)
    try:
        assert rec.nt == json.loads((path / "metadata.json").read_text())["theta_count"]
        assert np.array_equal(np.asarray(rec.u_edges), np.load(path / "u_edges.npy"))
    finally:
        close = getattr(rec, "close", None)
        if close:
            close()


def test_reference_reader_rejects_a_broken_record(tmp_path):
    """The reader is live, not a no-op: a record whose marginal CDF decreases is refused."""
    reader = reference_reader()
    if reader is None or not RECORDS:
        pytest.skip("reference checkout or fixture records not present")
    bad = tmp_path / "bad"
    shutil.copytree(RECORDS[0], bad)
    a = np.load(bad / "phi_cdf.npy")
    a[1], a[2] = a[2] + 1e-3, a[1]
    raw = (bad / "phi_cdf.npy").read_bytes()
    header = len(raw) - a.nbytes
    (bad / "phi_cdf.npy").write_bytes(raw[:header] + a.astype("<f8").tobytes())
    with pytest.raises(Exception):
        reader(bad, validate=True)
