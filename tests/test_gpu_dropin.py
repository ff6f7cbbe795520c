"""The drop-in from the reference's side: the reference solver itself
(oracle/_ref/dropin/oneflow_ref_ofg -- the reference built from its sources
with oracle/refbuild/ofg_adapter.cpp linked in and its task tables pointing
the hot-path task names at the adapter) runs the reference's own regression
cases with every task of TimeIntegral::Lusgs on the GPU through the C ABI,
and its output files must pass the reference's own regression comparison
(test/test.py: each file of autotest/test.txt line by line, every number
within 1e-8 of the golden file).  The cases and their golden files are copied
into oracle/_ref/cases by the reference build."""
import os
import re
import shutil
import subprocess
import tempfile

import pytest

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE = os.path.join(ROOT, "oracle", "_ref", "dropin", "oneflow_ref_ofg")
CASES = os.path.join(ROOT, "oracle", "_ref", "cases")
_NUM = re.compile(r"^[+-]?(\d+\.?\d*|\.\d+)([eE][+-]?\d+)?$")


def same_within(line1: str, line2: str, tol: float = 1e-8) -> bool:
    """test/test.py CmpFloatStr: numeric tokens within tol, others ignored."""
    a, b = line1.split(), line2.split()
    for x, y in zip(a, b):
        if _NUM.match(x) and _NUM.match(y) and abs(float(x) - float(y)) > tol:
            return False
    return True


def compare_files(got: str, want: str):
    """test/test.py CmpFile: returns None if equal, else the first bad line."""
    with open(got, encoding="utf-8-sig") as f1, open(want, encoding="utf-8-sig") as f2:
        for k, (l1, l2) in enumerate(zip(f1, f2)):
            if l1 != l2 and not same_within(l1, l2):
                return k, l1.rstrip(), l2.rstrip()
    return None


@pytest.mark.parametrize("case", ["plateuns2dslau2", "turbplateuns2droe_sa", "rae2822_roe_sa"])
def test_reference_regression_case_through_the_gpu_drop_in(case):
    src = os.path.join(CASES, case)
    if not (os.path.exists(EXE) and os.path.isdir(src)):
        pytest.skip("drop-in build absent (oracle/_ref/dropin: needs the reference sources at build time)")
    tmp = tempfile.mkdtemp(prefix="ofgdropin_")
    try:
        prj = os.path.join(tmp, case)
        shutil.copytree(src, prj)
        for sub in ("results", "log", "visual", "restart"):
            os.makedirs(os.path.join(prj, sub), exist_ok=True)
        r = subprocess.run([EXE, "0", case], cwd=tmp, stdout=subprocess.PIPE, stderr=subprocess.STDOUT,
                           timeout=1200)
        out = r.stdout.decode(errors="replace")
        assert r.returncode == 0, out[-3000:]
        assert "oneflow_b200: hot-path tasks on the GPU" in out   # the adapter ran, not the stock tasks
        with open(os.path.join(prj, "autotest", "test.txt"), encoding="utf-8-sig") as fh:
            files = [ln.strip() for ln in fh if ln.strip()]
        assert files
        for fn in files:
            got = os.path.join(prj, fn)
            want = os.path.join(prj, "autotest", os.path.basename(fn))
            assert os.path.exists(got), fn
            bad = compare_files(got, want)
            assert bad is None, (case, fn, bad)
    finally:
        shutil.rmtree(tmp, ignore_errors=True)


@pytest.mark.parametrize("name", ["cavity2d_quad", "cavity3d_hex"])
def test_incompressible_inner_iterations_through_the_gpu_drop_in(name):
    # The reference's incompressible solver (INsSolver, SIMPLE) with its
    # UPDATE_RESIDUALS task on the GPU (system/ins/function/funcMap.txt of the
    # drop-in build -> OfgInsUpdateResiduals -> ofg_ins_update_residuals):
    # the reference's own loop control, initialisation and output around it.
    # Its final state matches the reference's stock run (the fixture) within
    # 1e-9 of each field's magnitude, and every remax line matches the stock
    # run's to its six printed digits (a last-digit flip allowed).
    import numpy as np
    from golden_cases import build_ins
    from oracle_lib import run_ref_ins
    if not os.path.exists(EXE):
        pytest.skip("drop-in build absent (oracle/_ref/dropin: needs the reference sources at build time)")
    mesh, prm, wall, steps = build_ins(name)
    out = []
    dump, rem = run_ref_ins(mesh, prm, 1.0, steps, exe=EXE, output=out)
    assert "oneflow_b200: incompressible inner iterations on the GPU" in out[0]
    gold = np.load(os.path.join(ROOT, "tests", "golden", f"ins_{name}.npz"))
    for e in range(5):
        scale = max(np.abs(gold["q"][e]).max(), 1e-300)
        assert np.abs(dump["q"][e] - gold["q"][e]).max() / scale < 1e-9, e
    assert rem.shape == gold["remax_printed"].shape
    np.testing.assert_allclose(rem, gold["remax_printed"], rtol=6e-6, atol=0)
