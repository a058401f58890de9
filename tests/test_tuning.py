"""Tuning table parsing and the crossover setters (no GPU needed: they only
touch host-side state of the library)."""
from __future__ import annotations

import ctypes as C
import os

import pytest

from conftest import ROOT, load_recipe


@pytest.fixture(scope="module")
def bb():
    load_recipe("bigint_b200/build.py").build()
    import bigint_b200

    return bigint_b200


def _get(bb, key):
    v = C.c_uint64(0)
    assert bb.lib.bgpu_get_tuning(key, C.byref(v)) == 0
    return v.value


def test_set_get_roundtrip_and_limits(bb):
    old = _get(bb, bb.BGPU_TUNE_SCHOOLBOOK_MAX_LIMBS)
    assert bb.lib.bgpu_set_tuning(bb.BGPU_TUNE_SCHOOLBOOK_MAX_LIMBS, 96) == 0
    assert _get(bb, bb.BGPU_TUNE_SCHOOLBOOK_MAX_LIMBS) == 96
    assert bb.lib.bgpu_set_tuning(bb.BGPU_TUNE_SCHOOLBOOK_MAX_LIMBS, 257) == -1  # kernel limit 256
    assert bb.lib.bgpu_set_tuning(99, 1) == -1
    assert bb.lib.bgpu_set_tuning(bb.BGPU_TUNE_SCHOOLBOOK_MAX_LIMBS, old) == 0


def test_load_valid_table(bb, tmp_path):
    p = tmp_path / "t.txt"
    p.write_text("# comment\nsplit 20 8   # trailing comment\nbatch_split 18 7\nschoolbook_max_limbs 64\n"
                 "batch_schoolbook_max_limbs 128\nkaratsuba_max_limbs 300\nbatch_karatsuba_max_limbs 512\n"
                 "fft_min_limbs 0\nfft_max_limbs 0\n\n")
    old_split, old_bsplit = bb.get_split(20), bb.get_batch_split(18)
    assert bb.lib.bgpu_load_tuning(os.fsencode(str(p))) == 0
    assert bb.get_split(20) == 8
    assert bb.get_batch_split(18) == 7
    assert bb.get_split(18) != 7 or old_split == 7  # separate tables
    assert _get(bb, bb.BGPU_TUNE_SCHOOLBOOK_MAX_LIMBS) == 64
    assert _get(bb, bb.BGPU_TUNE_BATCH_SCHOOLBOOK_MAX_LIMBS) == 128
    assert _get(bb, bb.BGPU_TUNE_KARATSUBA_MAX_LIMBS) == 300
    assert _get(bb, bb.BGPU_TUNE_BATCH_KARATSUBA_MAX_LIMBS) == 512
    bb.set_split(20, 0)
    bb.set_batch_split(18, 0)
    assert bb.get_split(20) == old_split and bb.get_batch_split(18) == old_bsplit
    for k, v in ((bb.BGPU_TUNE_SCHOOLBOOK_MAX_LIMBS, 256), (bb.BGPU_TUNE_BATCH_SCHOOLBOOK_MAX_LIMBS, 256),
                 (bb.BGPU_TUNE_KARATSUBA_MAX_LIMBS, 0), (bb.BGPU_TUNE_BATCH_KARATSUBA_MAX_LIMBS, 0)):
        bb.set_tuning(k, v)


@pytest.mark.parametrize("body", ["bogus_key 3\n", "split 20 1\n", "split 30 9\n",
                                  "schoolbook_max_limbs 1000\n", "split 20\n", "batch_split 22 1\n",
                                  "karatsuba_max_limbs 513\n"])
def test_invalid_table_changes_nothing(bb, tmp_path, body):
    p = tmp_path / "bad.txt"
    p.write_text("schoolbook_max_limbs 32\n" + body)
    before = _get(bb, bb.BGPU_TUNE_SCHOOLBOOK_MAX_LIMBS)
    assert bb.lib.bgpu_load_tuning(os.fsencode(str(p))) == -1
    assert _get(bb, bb.BGPU_TUNE_SCHOOLBOOK_MAX_LIMBS) == before


def test_missing_file(bb):
    assert bb.lib.bgpu_load_tuning(b"/nonexistent/table.txt") == -1


def test_shipped_table_parses(bb):
    path = os.path.join(ROOT, "bigint_b200", "tuning_b200.txt")
    if not os.path.exists(path):
        pytest.skip("no shipped tuning table")
    assert bb.lib.bgpu_load_tuning(os.fsencode(path)) == 0
    for ln in range(10, 27):
        bb.lib.bgpu_set_split(ln, 0)
        bb.lib.bgpu_set_batch_split(ln, 0)
