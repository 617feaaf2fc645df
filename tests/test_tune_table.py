"""The autotuner's choice table on the host: set, get, save, load, clear
and argument checks (no device work)."""
import os

import pytest

import kronmult_b200 as kb


@pytest.fixture(autouse=True)
def _clean_table():
    kb.tune_clear()
    yield
    kb.tune_clear()


def test_set_get_clear():
    assert kb.tune_get(6, 4, "f64") == (None, 0)
    kb.tune_set(6, 4, "f64", "sq", 2)
    kb.tune_set(6, 4, "f32", "pipe")
    assert kb.tune_get(6, 4, "f64") == ("sq", 2)
    assert kb.tune_get(6, 4, "f32") == ("pipe", 0)
    assert kb.tune_get(6, 4, "split") == (None, 0)
    kb.tune_set(6, 4, "f64", None)
    assert kb.tune_get(6, 4, "f64") == (None, 0)
    kb.tune_clear()
    assert kb.tune_get(6, 4, "f32") == (None, 0)


def test_save_load_roundtrip(tmp_path):
    kb.tune_set(3, 8, "f64", "mma8")
    kb.tune_set(6, 6, "f64", "big", 4)
    kb.tune_set(5, 5, "split", "gen")
    path = os.path.join(tmp_path, "tune.txt")
    kb.tune_save(path)
    kb.tune_clear()
    kb.tune_load(path)
    assert kb.tune_get(3, 8, "f64") == ("mma8", 0)
    assert kb.tune_get(6, 6, "f64") == ("big", 4)
    assert kb.tune_get(5, 5, "split") == ("gen", 0)
    lines = open(path).read().split("\n")
    assert "6 6 0 5 4" in lines


def test_cluster_kernel_form_bits_roundtrip(tmp_path):
    """The "big" parameter carries the cluster size and the form bits (CUDA
    cores for FP64 n = 8, the intermediate in shared memory for FP64 n = 6)
    through the table and its file unchanged."""
    import re

    hdr = open(os.path.join(os.path.dirname(__file__), "..", "include", "kronmult.h")).read()
    defs = dict(re.findall(r"#define (KRON_BIG_\w+) (\d+)", hdr))
    assert int(defs["KRON_BIG_CUDA_CORES"]) == kb.BIG_CUDA_CORES
    assert int(defs["KRON_BIG_SMEM_W"]) == kb.BIG_SMEM_W
    kb.tune_set(6, 8, "f64", "big", 2 | kb.BIG_CUDA_CORES)
    kb.tune_set(6, 6, "f64", "big", kb.BIG_SMEM_W)
    path = os.path.join(tmp_path, "tune_bits.txt")
    kb.tune_save(path)
    kb.tune_clear()
    kb.tune_load(path)
    assert kb.tune_get(6, 8, "f64") == ("big", 2 | kb.BIG_CUDA_CORES)
    assert kb.tune_get(6, 6, "f64") == ("big", kb.BIG_SMEM_W)


@pytest.mark.parametrize("args", [
    (0, 4, 0, 3, 0), (7, 4, 0, 3, 0), (6, 0, 0, 3, 0), (6, 4, 3, 3, 0), (6, 4, 0, 9, 0),
    (6, 4, 0, 3, -1),
])
def test_set_rejects_bad_arguments(args):
    assert kb.lib().kron_tune_set(*args) == 1  # KRON_ERROR_INVALID_VALUE


def test_load_missing_file(tmp_path):
    rc = kb.lib().kron_tune_load(os.fsencode(os.path.join(tmp_path, "none.txt")))
    assert rc == 1  # KRON_ERROR_INVALID_VALUE
