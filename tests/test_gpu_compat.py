"""The reference-API layer (include/sfh_compat.hpp) against the reference.

oracle/_ref/compat_*/compat_check links the reference's own Fermions.cpp and
Lattice.cpp with libsfh.so and calls each function twice on the same inputs:
once the reference's definition, once the same-named sfh_compat:: one.  The
binary prints the relative differences; tolerances are those of the direct
C-ABI parity tests (operators and forces 1e-12; CG, whose stopping rule is
the reference's own 1e-12 relative residual, 1e-10; leapfrog trajectories
1e-10 on U and P)."""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

pytestmark = pytest.mark.gpu

DIMS = (4, 4, 4, 6)  # the lattice compat_check is built for


@pytest.fixture(scope="module")
def result(orc, tmp_path_factory):
    from oracle import build_ref
    exe = build_ref.compat_path()
    if not os.path.exists(exe):
        pytest.skip("compat_check was not built (needs the reference sources at build time)")
    d = tmp_path_factory.mktemp("compat")
    orc.random_gauge(DIMS, 0.3, 211).tofile(d / "U.bin")
    orc.random_momenta(DIMS, 212).tofile(d / "P.bin")
    orc.random_spinor(DIMS, 213).tofile(d / "phi.bin")
    r = subprocess.run([exe, str(d)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    line = [l for l in r.stdout.splitlines() if l.startswith("{")][-1]
    return json.loads(line)


@pytest.mark.parametrize("name,tol", [
    ("apply_DDdagger", 1e-12), ("solve_Y_field", 1e-12), ("solve_CG_DDdagger", 1e-10),
    ("compute_full_force_field", 1e-12), ("compute_fermion_only_force_field", 1e-12),
    ("compute_gauge_only_force_field", 1e-12), ("compute_Tr_P2", 1e-13), ("compute_action", 1e-12),
    ("compute_avg_plaq", 1e-12),
    ("apply_initial_step_to_conjugate_field.P", 1e-10), ("apply_intermediate_update.U", 1e-10),
    ("apply_intermediate_update.P", 1e-10), ("apply_final_step.U", 1e-10), ("apply_final_step.P", 1e-10),
    ("apply_final_step.X", 1e-9),
    ("local_leapfrog.U", 1e-10), ("local_leapfrog.P", 1e-10), ("local_leapfrog.X", 1e-9),
    ("local_leapfrog_fermion.U", 1e-10), ("local_leapfrog_fermion.P", 1e-10), ("local_leapfrog_fermion.X", 1e-9),
    ("local_leapfrog_gauge.U", 1e-12), ("local_leapfrog_gauge.P", 1e-12),
    ("precompute_polyakov_grid", 1e-12), ("correlator_over_fixed_distance_fast", 1e-12),
])
def test_compat_matches_reference(result, name, tol):
    assert result[name] < tol, (name, result[name])


def test_compat_hmc_update_runs(result):
    assert result["single_sweep.plaq_finite"] == 1.0


def test_compat_error_behaviour(result):
    """Fermions.cpp:714-716 and :609-614: std::runtime_error with the
    reference's messages."""
    assert result["non_hermitian.compat"].startswith("runtime_error")
    assert "P_pre is not Hermitian or not traceless" in result["non_hermitian.compat"]
    assert result["noconv.compat"].startswith("runtime_error")
    assert "failed to converge" in result["noconv.compat"]
