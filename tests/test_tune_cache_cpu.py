"""The tuned-plan cache file (lab_tune_cache_save / load / clear): host only, no GPU."""
import pytest

from linalglib_b200 import _lib as L


def _load(path):
    return L.lib().lab_tune_cache_load(str(path).encode())


def test_cache_file_round_trip(tmp_path):
    L.call("lab_tune_cache_clear")
    good = tmp_path / "good.txt"
    good.write_text("linalglib_b200 tune cache 1\n"
                    "spmv 390915 390915 16070499 0 2 8 0 49.4\n"
                    "spmv 59835 59835 8587063 0 2 16 2 12.5\n"
                    "gemm 2097152 2097152 14581760 2097152 390915 9022412 1 1 2 2310.0\n")
    assert _load(good) == L.LAB_OK
    out = tmp_path / "out.txt"
    L.call("lab_tune_cache_save", str(out).encode())
    lines = out.read_text().splitlines()
    assert lines[0] == "linalglib_b200 tune cache 1"
    assert any(l.startswith("spmv 390915 390915 16070499 0 2 8 0") for l in lines)
    assert any(l.startswith("spmv 59835 59835 8587063 0 2 16 2") for l in lines)  # halo form
    assert any(l.startswith("gemm 2097152 2097152 14581760 2097152 390915 9022412 1 1 2")
               for l in lines)
    L.call("lab_tune_cache_clear")
    L.call("lab_tune_cache_save", str(out).encode())
    assert out.read_text().splitlines() == ["linalglib_b200 tune cache 1"]


@pytest.mark.parametrize("text", [
    "not a cache\n",
    "linalglib_b200 tune cache 1\nspmv 10 10 30 0 2 3 0 1.0\n",        # 3 lanes
    "linalglib_b200 tune cache 1\nspmv 10 10 30 0 7 8 0 1.0\n",        # unknown schedule
    "linalglib_b200 tune cache 1\nspmv 10 10 30 0 2 8 3 1.0\n",        # unknown VECTOR form
    "linalglib_b200 tune cache 1\ngemm 1 2 3 2 4 5 3 3 4 1.0\n",       # sym 3
    "linalglib_b200 tune cache 1\ngemm 1 2 3 2 4 5 2 2 3 1.0\n",       # fill 2/3
    "linalglib_b200 tune cache 1\nsomething else\n",
])
def test_cache_file_refused(tmp_path, text):
    L.call("lab_tune_cache_clear")
    bad = tmp_path / "bad.txt"
    bad.write_text(text)
    assert _load(bad) == L.LAB_BAD_ARG
    out = tmp_path / "after.txt"
    L.call("lab_tune_cache_save", str(out).encode())
    assert out.read_text().splitlines() == ["linalglib_b200 tune cache 1"]  # nothing loaded


def test_cache_missing_file(tmp_path):
    assert _load(tmp_path / "none.txt") == L.LAB_BAD_ARG
