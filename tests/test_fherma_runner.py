"""The drop-in boundary: fherma_init / fherma_run / fherma_free
(libfherma_polymul.so) driven through point directories, the way the
reference's own end-to-end test drives its solution (tests/validate.py:64-101:
make a point directory, run the solution binary, compare c.bin bytes).

Two harnesses run the same points: polymul_solution (this repository's runner)
and, when it was built (oracle/_ref/fherma_main), the reference's own main.cpp
compiled unmodified against libfherma_polymul.so."""
import json
import os
import subprocess

import pytest

from tests.golden.cases import load_golden, point_cases, sha

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "fherma-polymul-baseline_b200")
RUNNER = os.path.join(PKG, "polymul_solution")
SHIM = os.path.join(PKG, "libfherma_polymul.so")
REF_MAIN = os.path.join(ROOT, "oracle", "_ref", "fherma_main")


def make_point_dir(tmp, point, corrupt=None):
    """Writes the bundle layout; `corrupt` = case index whose a.bin is truncated."""
    n, L = point["N"], point["L"]
    q = int(point["q"], 16)
    os.makedirs(os.path.join(tmp, "point"), exist_ok=True)
    with open(os.path.join(tmp, "point", "q.bin"), "wb") as f:
        f.write(q.to_bytes(4 * L, "little"))
    expected = []
    for idx, (label, a, b, rec) in enumerate(point_cases(point)):
        d = os.path.join(tmp, "cases", f"{idx:06d}")
        os.makedirs(d, exist_ok=True)
        with open(os.path.join(d, "a.bin"), "wb") as f:
            f.write(a.tobytes()[: 100] if idx == corrupt else a.tobytes())
        with open(os.path.join(d, "b.bin"), "wb") as f:
            f.write(b.tobytes())
        expected.append(rec["c_sha256"])
    with open(os.path.join(tmp, "manifest.json"), "w") as f:
        json.dump({"point": {"N": n, "W": point["W"], "L": L}, "cases": len(expected)}, f)
    return expected


def verify(tmp, expected, crashed=()):
    results = json.load(open(os.path.join(tmp, "out", "results.json")))
    assert results["init_s"] >= 0 and len(results["cases"]) == len(expected)
    for idx, want in enumerate(expected):
        rec = results["cases"][idx]
        assert rec["i"] == idx
        if idx in crashed:
            assert rec["status"] == "crashed" and rec["seconds"] is None
            continue
        assert rec["status"] == "ok" and rec["seconds"] > 0, rec
        with open(os.path.join(tmp, "out", f"{idx:06d}", "c.bin"), "rb") as f:
            assert sha(f.read()) == want, f"case {idx}"


def test_shim_exports_the_reference_signatures():
    out = subprocess.run(["nm", "-DC", "--defined-only", SHIM], capture_output=True, text=True, check=True).stdout
    assert "fherma_init(fherma::Point const&)" in out
    assert "fherma_run(void*, fherma::Inputs const&)" in out
    assert "fherma_free(void*)" in out


def test_runner_usage_and_missing_point(tmp_path):
    assert subprocess.run([RUNNER], capture_output=True).returncode == 2
    r = subprocess.run([RUNNER, str(tmp_path)], capture_output=True, text=True)
    assert r.returncode == 1 and "manifest.json" in r.stderr


HARNESSES = [RUNNER] + ([REF_MAIN] if os.path.exists(REF_MAIN) else [])


@pytest.mark.gpu
@pytest.mark.parametrize("harness", HARNESSES, ids=lambda p: os.path.basename(p))
@pytest.mark.parametrize("which", [(32, None), (32, 1), (1024, None), (32768, None)])
def test_point_directories(cuda, tmp_path, harness, which):
    n, delta = which
    point = [p for p in load_golden()["points"] if p["N"] == n and p["delta"] == delta][0]
    expected = make_point_dir(str(tmp_path), point)
    subprocess.run([harness, str(tmp_path)], check=True, timeout=600)
    verify(str(tmp_path), expected)


@pytest.mark.gpu
def test_crashed_case_is_recorded_and_run_continues(cuda, tmp_path):
    point = [p for p in load_golden()["points"] if p["N"] == 32 and p["delta"] is None][0]
    expected = make_point_dir(str(tmp_path), point, corrupt=3)
    subprocess.run([RUNNER, str(tmp_path)], check=True, timeout=600)
    verify(str(tmp_path), expected, crashed={3})
