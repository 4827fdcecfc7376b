#!/usr/bin/env python3
"""Build the reference's own sources into oracle/_ref/ (test infrastructure).

The reference (alexanderchasteen/Staggered_Fermions_HMC) fixes the lattice
size, the fermion mass and the CG tolerance as compile-time constants in its
Parameters.h (Parameters.h:9-24) and needs Eigen, which is absent here.  This
recipe therefore builds one binary per (L, T, mass, tol) in a directory of
symbolic links to the unmodified reference files, next to:

  * a generated Parameters.h with the same constant names, and
  * the project's Eigen-API subset header (oracle/eigen_subset).

Only Lattice.cpp, Fermions.cpp, SU3_Sampling.cpp and rng.cpp are compiled,
together with oracle/ref_harness.cpp, and once more with
oracle/compat_check.cpp and libsfh.so (the side-by-side check of the
reference-API layer).  Outputs go to oracle/_ref/ only.
Nothing here runs the reference's own build (submit_roar.slurm).

usage: python oracle/build_ref.py --reference DIR [L T mass tol] ...
       (DIR: a checkout of the reference; or set SFH_REFERENCE_DIR.  Without
       L T mass tol the fixture and benchmark set is built.)
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
# the reference checkout: --reference DIR on the command line, else the
# SFH_REFERENCE_DIR environment variable; None = not available
REF = os.environ.get("SFH_REFERENCE_DIR") or None


def set_reference(path):
    global REF
    REF = path
OUT = os.path.join(HERE, "_ref")
SOURCES = ["Lattice.cpp", "Fermions.cpp", "SU3_Sampling.cpp", "rng.cpp"]
HEADERS = ["Lattice.h", "Fermions.h", "SU3_Sampling.h", "rng.h"]

# (L, T, mass, tol): the golden-fixture lattices, then the uneven-batch
# benchmark lattices {8^4, 12^4, 16^4, 16^3x32} x masses {0.05, 0.1, 0.2}
DEFAULT_CONFIGS = [
    (4, 4, 0.1, 1e-12),
    (4, 6, 0.5, 1e-12),
] + [(L, T, m, 1e-10) for (L, T) in ((8, 8), (12, 12), (16, 16), (16, 32))
     for m in (0.05, 0.1, 0.2)]


def tag(L, T, mass, tol):
    return f"L{L}T{T}_m{mass:g}_tol{tol:g}"


def parameters_h(L, T, mass, tol, maxit=50000, eps=1e-2, nsteps=100):
    """Generated stand-in for the reference Parameters.h (same names)."""
    V = L * L * L * T
    return f"""// generated by oracle/build_ref.py: lattice {L}^3x{T}, mass {mass!r}, tol {tol!r}
#pragma once
#include <vector>
#include <array>
#include <cmath>
#include <random>
constexpr int Spatial_Size = {L};
constexpr int temporal_size = {T};
constexpr int array_size = 4*Spatial_Size*Spatial_Size*Spatial_Size*18*temporal_size;
constexpr int Nplaq = Spatial_Size*Spatial_Size*Spatial_Size*temporal_size*6;
const int maxdistance = std::floor(Spatial_Size/2)-1;
const double fermion_mass = {mass!r};
const int Staggered_Fermion_field_indices = {6 * V};
const int conjugate_field_array_size = {72 * V};
const double epsilon = {eps!r};
const int number_of_steps_fermion = {nsteps};
const double tol = {tol!r};
const int max_iter = {maxit};
constexpr double dbeta = 0.5;
constexpr double beta_min = 4.1;
constexpr int CONFIG = 1;
constexpr double beta_max = beta_min + CONFIG * dbeta;
constexpr std::array<double, CONFIG> make_couplings() {{
    std::array<double, CONFIG> a{{}};
    for (int i = 0; i < CONFIG; ++i) a[i] = beta_min + i * dbeta;
    return a;
}}
inline std::array<double, CONFIG> coupling_constants = make_couplings();
constexpr int thermal_sweeps = 1000;
constexpr int autocorrelation_sweeps = 100;
constexpr int measurment_sweeps = 1000;
constexpr int maxlag = 10;
constexpr double c_11 = 5.0/3.0;
constexpr double c_12 = -1.0/12.0;
"""


def build(L, T, mass, tol, verbose=True):
    d = os.path.join(OUT, tag(L, T, mass, tol))
    exe = os.path.join(d, "ref_harness")
    os.makedirs(d, exist_ok=True)
    for f in SOURCES + HEADERS:
        link = os.path.join(d, f)
        if not os.path.lexists(link):
            os.symlink(os.path.join(REF, f), link)
    with open(os.path.join(d, "Parameters.h"), "w") as fh:
        fh.write(parameters_h(L, T, mass, tol))
    harness = os.path.join(d, "ref_harness.cpp")
    if not os.path.lexists(harness):
        os.symlink(os.path.join(HERE, "ref_harness.cpp"), harness)
    cmd = ["g++", "-std=c++17", "-O3", "-fopenmp", "-w",
           "-I" + os.path.join(HERE, "eigen_subset"), "-I" + d, "-o", exe]
    cmd += [os.path.join(d, f) for f in SOURCES] + [harness]
    if verbose:
        print("build", tag(L, T, mass, tol), flush=True)
    subprocess.run(cmd, check=True)
    # keep only the binary and the generated header: the links point into the
    # reference tree, which does not travel with the repository
    for f in SOURCES + HEADERS + ["ref_harness.cpp"]:
        os.remove(os.path.join(d, f))
    return exe


# (L, T, mass, tol, eps, nsteps) of the reference-API layer check: a short
# production trajectory (global step size and count) on a 4^3x6 lattice
COMPAT_CONFIG = (4, 6, 0.2, 1e-12, 0.02, 4)
COMPAT_SOURCES = [os.path.join(HERE, "compat_check.cpp"),
                  os.path.join(os.path.dirname(HERE), "include", "sfh_compat.hpp")]


def compat_path():
    L, T, mass, tol, eps, nsteps = COMPAT_CONFIG
    return os.path.join(OUT, "compat_" + tag(L, T, mass, tol), "compat_check")


def build_compat(verbose=True):
    """Reference sources + oracle/compat_check.cpp, linked with libsfh.so
    (found at run time through an rpath relative to the binary)."""
    L, T, mass, tol, eps, nsteps = COMPAT_CONFIG
    exe = compat_path()
    d = os.path.dirname(exe)
    root = os.path.dirname(HERE)
    pkg = os.path.join(root, "staggered_fermions_hmc_b200")
    lib = os.path.join(pkg, "libsfh.so")
    if not os.path.exists(lib):
        raise RuntimeError("build libsfh.so first")
    if os.path.exists(exe) and all(os.path.getmtime(exe) >= os.path.getmtime(f) for f in COMPAT_SOURCES):
        return exe
    os.makedirs(d, exist_ok=True)
    for f in SOURCES + HEADERS:
        link = os.path.join(d, f)
        if not os.path.lexists(link):
            os.symlink(os.path.join(REF, f), link)
    with open(os.path.join(d, "Parameters.h"), "w") as fh:
        fh.write(parameters_h(L, T, mass, tol, eps=eps, nsteps=nsteps))
    rpath = "$ORIGIN/" + os.path.relpath(pkg, d)
    cmd = ["g++", "-std=c++17", "-O2", "-fopenmp", "-w",
           "-I" + os.path.join(HERE, "eigen_subset"), "-I" + d, "-I" + os.path.join(root, "include"),
           "-o", exe] + [os.path.join(d, f) for f in SOURCES] + [COMPAT_SOURCES[0]]
    cmd += ["-L" + pkg, "-lsfh", "-Wl,-rpath," + rpath]
    if verbose:
        print("build compat_check", flush=True)
    try:
        subprocess.run(cmd, check=True)
    finally:
        for f in SOURCES + HEADERS:
            os.remove(os.path.join(d, f))
    return exe


# the reference's HEX staple steps (apply_step_1/3/5 of Smearing.cpp) on a
# 4^4 lattice: the golden fixture for the smearing restatement
HEX_LT = (4, 4)


def hex_path():
    L, T = HEX_LT
    return os.path.join(OUT, f"hex_L{L}T{T}", "hex_harness")


def build_hex(verbose=True):
    """Reference sources + the unmodified Smearing.cpp + oracle/hex_harness.cpp.
    Smearing.h (included first by Smearing.cpp) uses Parameters.h and
    Lattice.h names before including anything (Smearing.h:11), so that one
    file is compiled with those two headers forced in front (-include); no
    source is changed."""
    L, T = HEX_LT
    exe = hex_path()
    d = os.path.dirname(exe)
    src = os.path.join(HERE, "hex_harness.cpp")
    if os.path.exists(exe) and os.path.getmtime(exe) >= os.path.getmtime(src):
        return exe
    os.makedirs(d, exist_ok=True)
    files = SOURCES + HEADERS + ["Smearing.cpp", "Smearing.h"]
    for f in files:
        link = os.path.join(d, f)
        if not os.path.lexists(link):
            os.symlink(os.path.join(REF, f), link)
    with open(os.path.join(d, "Parameters.h"), "w") as fh:
        fh.write(parameters_h(L, T, 0.1, 1e-12))
    base = ["g++", "-std=c++17", "-O2", "-fopenmp", "-w", "-I" + os.path.join(HERE, "eigen_subset"), "-I" + d]
    smear_o = os.path.join(d, "Smearing.o")
    if verbose:
        print("build hex_harness", flush=True)
    try:
        subprocess.run(base + ["-include", os.path.join(d, "Parameters.h"), "-include", os.path.join(d, "Lattice.h"),
                               "-c", os.path.join(d, "Smearing.cpp"), "-o", smear_o], check=True)
        subprocess.run(base + ["-o", exe] + [os.path.join(d, f) for f in SOURCES] + [src, smear_o], check=True)
    finally:
        for f in files:
            os.remove(os.path.join(d, f))
        if os.path.exists(smear_o):
            os.remove(smear_o)
    return exe


def exe_path(L, T, mass, tol):
    return os.path.join(OUT, tag(L, T, mass, tol), "ref_harness")


def main(argv):
    argv = list(argv)
    if "--reference" in argv:
        k = argv.index("--reference")
        set_reference(argv[k + 1])
        del argv[k:k + 2]
    if not REF or not os.path.isdir(REF):
        print(f"reference sources not found ({REF!r}; give --reference DIR or set SFH_REFERENCE_DIR); "
              "nothing to build")
        return 0
    configs = DEFAULT_CONFIGS
    if len(argv) >= 4:
        configs = []
        for i in range(0, len(argv) - 3, 4):
            configs.append((int(argv[i]), int(argv[i + 1]), float(argv[i + 2]), float(argv[i + 3])))
    import concurrent.futures as cf
    todo = [c for c in configs if not os.path.exists(exe_path(*c))]
    with cf.ThreadPoolExecutor(max_workers=max(1, min(8, os.cpu_count() or 1))) as ex:
        list(ex.map(lambda c: build(*c), todo))
    if len(argv) < 4:
        build_compat()
        build_hex()
    return 0


if __name__ == "__main__":
    sys.exit(main(sys.argv[1:]))
