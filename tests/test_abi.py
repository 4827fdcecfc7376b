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
