"""Host side of the plain DB pass (irisb200.scan.PlainScan over the library's
irs_scan_*), no GPU: the native candidate list equals the batch autotuner's,
the chunking covers the DB, and bad configurations are refused before any
engine is touched.  The handles are placeholders: these calls only store them."""
from __future__ import annotations

import pytest

import irisb200
from irisb200.batched import BatchedEngine
from irisb200.scan import PlainScan


class _H:
    def __init__(self, v):
        self.h = v


def _scan(n_slots=64, db_len=100_000):
    return PlainScan(_H(1), [_H(10 + p) for p in range(3)], [_H(20 + p) for p in range(3)], _H(3), _H(2),
                     n_slots, db_len)


@pytest.mark.parametrize("n_slots,db_len", [(64, 524_288), (20, 524_288), (8, 2000), (2, 1000), (160, 100_000)])
def test_native_candidates_match_the_batch_autotuner(n_slots, db_len):
    ps = _scan(n_slots, db_len)
    try:
        assert ps.candidates() == BatchedEngine._candidates(n_slots * 32, db_len)
    finally:
        ps.close()


def test_default_configuration_and_chunks():
    ps = _scan(64, 100_000)
    try:
        assert ps.cand == ("split", 0, 65536)
        assert ps.chunks() == [(0, 65536), (65536, 34464)]
    finally:
        ps.close()


def test_bad_configurations_are_refused():
    ps = _scan()
    try:
        for cand in (("pair", 128, 32768), ("split", 256, 1000), ("split", 256, 0)):
            with pytest.raises(irisb200.IrisError):
                ps.configure(cand)
        assert ps.cand == ("split", 0, 65536)
        with pytest.raises(ValueError):
            ps.configure(("other", 256, 32768))
    finally:
        ps.close()
