"""Package boundary: PyTorch appears only in the gpk package (python/gpk),
which carries the reference's python/gpk names (GPKGrid, ThermoModel,
SolidificationThermo; albert-hzbn/GPK python/gpk/__init__.py) and the
torch.autograd.Function of the adjoint; the gpk_b200 binding of the C ABI
imports NumPy only."""
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _run(code):
    r = subprocess.run([sys.executable, "-c", code], cwd=ROOT, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    return r.stdout.strip()


def test_binding_does_not_import_torch():
    out = _run("import sys; sys.path.insert(0, '.'); import gpk_b200, gpk_b200.sweep, gpk_b200.batch; "
               "print('torch' in sys.modules)")
    assert out == "False"


def test_gpk_package_names():
    out = _run("import sys; sys.path[:0] = ['python']; import gpk, torch; "
               "print(gpk.GPKGrid.__name__, issubclass(gpk.GPKLoss, torch.autograd.Function), "
               "gpk.SolidificationThermo().model, gpk.ThermoModel(sigma0=0.25).sigma0)")
    assert out == "GPKGrid True solidification 0.25"
