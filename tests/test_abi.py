"""The C-ABI library loads without a GPU and exports every entry point that
include/*.h declares, and the Python binding covers exactly that set."""
import ctypes
import glob
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"\b(sfh_[a-z0-9_]+)\s*\(", text):
            names.add(m.group(1))
    return names


def test_header_declares_entry_points():
    names = declared_symbols()
    assert {"sfh_create", "sfh_dirac", "sfh_ddag", "sfh_cg_solve", "sfh_batch_solve"} <= names


def test_library_exports_every_declared_symbol():
    import staggered_fermions_hmc_b200 as sfh
    lib = ctypes.CDLL(sfh.LIB_PATH)
    missing = [n for n in sorted(declared_symbols()) if not hasattr(lib, n)]
    assert not missing, missing


def test_binding_covers_header():
    import staggered_fermions_hmc_b200 as sfh
    assert set(sfh.SIGNATURES) == declared_symbols()


def test_status_strings_without_gpu():
    import staggered_fermions_hmc_b200 as sfh
    lib = sfh.load_library()
    assert lib.sfh_version() >= 1
    assert b"converge" in lib.sfh_status_string(sfh.SFH_ERR_NOCONV)


def test_fastdiv_host_emulation():
    """The magic-number division used for coordinates (sfh_core.cuh FastDiv),
    emulated in Python, equals floor division for every divisor used."""
    def fastdiv(n, d):
        l = 0
        while (1 << l) < d:
            l += 1
        if l == 0:
            return n
        m = ((((1 << l) - d) << 32) // d + 1) & 0xFFFFFFFF
        t = (m * n) >> 32
        return (t + ((n - t) >> 1)) >> (l - 1)
    import random
    rnd = random.Random(5)
    for d in list(range(1, 130)) + [192, 256, 1000]:
        for n in [0, 1, d - 1, d, d + 1, 2 ** 31 - 1, 2 ** 28] + [rnd.randrange(2 ** 31) for _ in range(200)]:
            assert fastdiv(n, d) == n // d, (n, d)


COMPAT_FUNCTIONS = [
    "configure", "settings", "shutdown", "apply_DDdagger", "solve_CG_DDdagger", "solve_X_field", "solve_Y_field",
    "compute_full_force_field", "compute_fermion_only_force_field", "compute_gauge_only_force_field",
    "compute_Tr_P2", "generate_phi_field", "generate_conjugate_field_configuration",
    "apply_initial_step_to_conjugate_field", "apply_intermediate_update_to_gauge_field_and_conjugate_field",
    "apply_final_step", "Monte_carlo_step", "single_sweep_monte_carlo_update_WITH_FERMIONS",
    "local_initial_half_step", "local_leapfrog_steps", "local_final_step", "local_initial_half_step_fermion",
    "local_leapfrog_steps_fermion", "local_final_step_fermion", "local_initial_half_step_gauge",
    "local_leapfrog_steps_gauge", "local_final_step_gauge", "compute_action", "compute_avg_plaq",
    "precompute_polyakov_grid", "correlator_over_fixed_distance_fast", "save_lattice_configs",
    "load_lattice_configs", "Apply_HEX_smearing", "Apply_4HEX_smearing", "heatbath_update",
]


def test_compat_header_declares_and_library_defines():
    """include/sfh_compat.hpp compiles on its own and every function it
    declares is defined in libsfh.so (no GPU needed)."""
    import shutil
    import subprocess
    import staggered_fermions_hmc_b200 as sfh
    hdr = os.path.join(ROOT, "include", "sfh_compat.hpp")
    text = open(hdr).read()
    for name in COMPAT_FUNCTIONS:
        assert re.search(r"\b" + name + r"\(", text), name
    gxx = shutil.which("g++")
    if gxx:
        r = subprocess.run([gxx, "-std=c++17", "-fsyntax-only", "-x", "c++", "-I" + os.path.join(ROOT, "include"),
                            hdr], capture_output=True, text=True)
        assert r.returncode == 0, r.stderr
    nm = shutil.which("nm")
    if nm:
        out = subprocess.run([nm, "-DC", "--defined-only", sfh.LIB_PATH], capture_output=True, text=True).stdout
        missing = [n for n in COMPAT_FUNCTIONS if "sfh_compat::" + n + "(" not in out]
        assert not missing, missing


def test_python_constants_match_header():
    """Every #define of include/sfh.h with a number has the same value in the
    binding (SFH_ERR_* by name, SFH_PREC_* as PREC_*, the others without the
    SFH_ prefix)."""
    import staggered_fermions_hmc_b200 as sfh
    text = open(os.path.join(ROOT, "include", "sfh.h")).read()
    defines = {m.group(1): int(m.group(2)) for m in re.finditer(r"#define (SFH_[A-Z0-9_]+) (\d+)", text)}
    assert "SFH_PREC_BF16" in defines
    for name, value in defines.items():
        py = name if name.startswith(("SFH_OK", "SFH_ERR_")) else name[len("SFH_"):]
        assert getattr(sfh, py) == value, (name, py)
    assert sorted(sfh.PRECISIONS.values()) == sorted(v for k, v in defines.items() if k.startswith("SFH_PREC_"))


def test_null_handles_rejected_without_a_gpu():
    """Entry points check their handle before any CUDA call: a null context
    or batch gives SFH_ERR_INVALID (the staged Dslash storages, its test
    hook and the schedules among them)."""
    import staggered_fermions_hmc_b200 as sfh
    lib = sfh.load_library()
    buf = (ctypes.c_double * 8)()
    assert lib.sfh_set_staging_fault(None, 0) == sfh.SFH_ERR_INVALID
    assert lib.sfh_dslash_storage(None, 6, buf, buf) == sfh.SFH_ERR_INVALID
    assert lib.sfh_set_schedule(None, 2, 4, 7) == sfh.SFH_ERR_INVALID
    assert lib.sfh_batch_set_schedule(None, 2, 4, 6) == sfh.SFH_ERR_INVALID
    assert lib.sfh_batch_set_hop_widths(None, 4, 2) == sfh.SFH_ERR_INVALID
