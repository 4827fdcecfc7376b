"""The bench's algorithmic-byte accounting (the basis of every roofline
figure it reports), checked on CPU against hand counts for small specs."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def _info(iters, nru):
    return {"iters_parity": [iters, iters], "reliable_updates": nru}


def test_kernel_bytes_fp64_one_rhs():
    """FP64, one system with one RHS: per parity and iteration hop1 reads p and
    writes t (2 spinors), hop2 reads t, p, r and writes v (4), update moves 5
    spinors and 2 solution vectors; both hops read the 8 links of every output
    site once."""
    import bench
    dims = (4, 4, 4, 4)
    Vh = 128
    spec = [{"dims": dims, "nrhs": 1}]
    out = bench.kernel_bytes(spec, [[_info(10, 0)]], "f64")
    s, sx, lb = 48, 48, 144
    per_parity = {"cg_hop1": 10 * Vh * (2 * s + 8 * lb),
                  "cg_hop2": 10 * Vh * (4 * s + 8 * lb),
                  "cg_update": 10 * Vh * (5 * s + 2 * sx)}
    for k, v in per_parity.items():
        assert out[k] == pytest.approx(2 * v), k


def test_kernel_bytes_links_shared_by_rhs_and_reliable_updates():
    """FP16, two RHS of one system: links are counted once per (system,
    parity, iteration) with the longer lane's count, spinors per RHS; each
    reliable update adds an FP64 hop to both hop kernels (or to the two
    reliable-update kernels of the system-blocked schedule), the second with
    the search direction rebuilt.  The increment x_lo is FP32."""
    import bench
    dims = (4, 4, 4, 8)
    Vh = 256
    spec = [{"dims": dims, "nrhs": 2}]
    infos = [[_info(12, 2), _info(20, 4)]]
    out = bench.kernel_bytes(spec, infos, "f16")
    s, sx, lb = 16, 24, 24
    its = 12 + 20
    nru = (2 + 4) / 2.0  # per parity
    ru1 = nru * Vh * (8 * 144 + 48 + sx + 48)
    ru2 = nru * Vh * (8 * 144 + 48 + 2 * 48 + 2 * sx + 48 + s + 3 * s)
    hop1 = its * Vh * 2 * s + 20 * 8 * lb * Vh
    hop2 = its * Vh * 4 * s + 20 * 8 * lb * Vh
    upd = its * Vh * (5 * s + 2 * sx)
    assert out["cg_hop1"] == pytest.approx(2 * (hop1 + ru1))
    assert out["cg_hop2"] == pytest.approx(2 * (hop2 + ru2))
    assert out["cg_update"] == pytest.approx(2 * upd)
    assert bench.solve_bytes(spec, infos, "f16") == pytest.approx(2 * (hop1 + hop2 + upd + ru1 + ru2))
    sep = bench.kernel_bytes(spec, infos, "f16", ru_separate=True)
    assert sep["cg_hop1"] == pytest.approx(2 * hop1) and sep["cg_ru1"] == pytest.approx(2 * ru1)
    assert sep["cg_hop2"] == pytest.approx(2 * hop2) and sep["cg_ru2"] == pytest.approx(2 * ru2)
    assert sum(sep.values()) == pytest.approx(sum(out.values()))


def test_dslash_bytes_table():
    """Per output site of one hop: 8 links, one input and one output vector."""
    import bench
    link = {0: 144, 1: 48, 2: 24, 3: 72, 4: 24, 5: 96, 6: 24, 7: 24}
    vec = {0: 48, 1: 24, 2: 16, 3: 24, 4: 16, 5: 48, 6: 16, 7: 16}
    for st in link:
        assert bench.DSLASH_BYTES[st] == 8 * link[st] + 2 * vec[st], bench.DSLASH_NAMES[st]


def test_batch_spec_is_the_seeded_workload():
    """64 systems from the stated sets, 1-8 RHS each, reproducible."""
    import bench
    a, b = bench.batch_spec(), bench.batch_spec()
    assert a == b and len(a) == 64
    assert all(s["dims"] in bench.LATTICES and s["mass"] in bench.MASSES and s["eps"] in bench.EPSES
               and 1 <= s["nrhs"] <= 8 for s in a)
    assert sum(s["nrhs"] for s in a) == 296


def test_batch_classes_cover_the_batch():
    """The reference sample's strata: (lattice, mass, eps) classes, with every
    solve of the batch in exactly one class."""
    import bench
    spec = bench.batch_spec()
    classes = bench.batch_classes(spec)
    assert len(classes) <= 24 and len({c[0] for c in classes}) == len(classes)
    assert sum(c[2] for c in classes) == 296
    for key, k, n in classes:
        assert (tuple(spec[k]["dims"]), spec[k]["mass"], spec[k]["eps"]) == key
        assert n == sum(s["nrhs"] for s in spec if (tuple(s["dims"]), s["mass"], s["eps"]) == key)


def test_cpu_estimate_weights_classes_by_their_solves(tmp_path):
    """solves/s = sum of the sampled classes' solves / sum n_c * mean t_c."""
    import bench
    spec = [{"dims": (4, 4, 4, 4), "mass": 0.1, "eps": 0.3, "nrhs": 3, "gauge_seed": 1, "rhs_seed": 2},
            {"dims": (4, 4, 4, 8), "mass": 0.2, "eps": 1.0, "nrhs": 1, "gauge_seed": 3, "rhs_seed": 4},
            {"dims": (4, 4, 4, 4), "mass": 0.1, "eps": 0.3, "nrhs": 2, "gauge_seed": 5, "rhs_seed": 6}]
    s = bench.CpuSampler(spec, str(tmp_path))
    assert [c[2] for c in s.classes] == [5, 1]
    est = s.estimate([(0, 1.0, "reference"), (0, 3.0, "reference"), (1, 10.0, "port")])
    assert est["value"] == pytest.approx(6 / (5 * 2.0 + 1 * 10.0))
    assert est["kind"] == "mixed" and est["reference_solves"] == 2 and est["port_solves"] == 1
    assert est["batch_cpu_seconds_estimate"] == pytest.approx(20.0)
    partial = s.estimate([(1, 10.0, "port")])
    assert partial["classes_timed"] == 1 and partial["value"] == pytest.approx(0.1)


def test_reference_arm_is_cpu_only_and_reports_the_same_workload(monkeypatch, capsys):
    """The reference arm builds its inputs with the oracle's generators and
    times CPU solves only: the library is never imported, the config equals
    the GPU arm's, and ms_per_step is the measured step time."""
    import json
    import sys

    import bench
    for k in ("RANK", "WORLD_SIZE", "LOCAL_RANK"):
        monkeypatch.delenv(k, raising=False)
    spec = [{"dims": (8, 8, 8, 8), "mass": m, "eps": 0.3, "nrhs": 2, "gauge_seed": 10 + i,
             "rhs_seed": 100 + i} for i, m in enumerate((0.2, 0.1))]

    class Args:
        warmup, steps, gpus, ref_budget = 1, 2, 1, 0.01
    loaded_before = "staggered_fermions_hmc_b200" in sys.modules
    bench.run_reference_arm(Args(), spec)
    line = json.loads(capsys.readouterr().out.strip().splitlines()[-1])
    if not loaded_before:
        assert "staggered_fermions_hmc_b200" not in sys.modules
    assert line["impl"] == "reference" and line["config"] == bench.workload_config(spec, 1)
    assert line["cpu_baseline"]["kind"] in ("reference", "port", "mixed")
    assert line["reference_sample"]["solves_timed"] >= 2
    assert line["value"] > 0 and 0 < line["ms_per_step"] < 60000


def test_e2e_pipeline_order():
    """The pipelined end-to-end measurement: every step uploads, solves and
    downloads on its own batch (n % 2); a batch's solutions are downloaded
    before its next inputs are uploaded, and a step's upload happens before
    its solve."""
    import threading
    import types

    import bench

    log, lock = [], threading.Lock()

    class FakeBatch:
        def __init__(self, name):
            self.name, self.stream = name, 0

        def solve(self, tol, max_iter):
            with lock:
                log.append(("solve", self.name))

    class Ev:
        def __init__(self, enable_timing=False):
            pass

        def record(self, s):
            pass

        def synchronize(self):
            pass

        def elapsed_time(self, other):
            return 100.0

    fake_torch = types.SimpleNamespace(cuda=types.SimpleNamespace(
        synchronize=lambda: None, ExternalStream=lambda p: p, Event=Ev))

    def upload(X):
        with lock:
            log.append(("up", X.name))

    def download(X):
        with lock:
            log.append(("down", X.name))

    pair = (FakeBatch("A"), FakeBatch("B"))
    steps = 5
    ms = bench.e2e_pipelined(fake_torch, pair, upload, download, steps)
    assert ms == 100.0 / steps
    timed = log[6:]  # after the warm-up: up, solve, down for each batch
    assert log[:6] == [("up", "A"), ("solve", "A"), ("down", "A"), ("up", "B"), ("solve", "B"), ("down", "B")]
    for op in ("up", "solve", "down"):
        assert sum(1 for o, _ in timed if o == op) == steps
    # per batch, the operations come in the order up, solve, down, up, ...
    for name in ("A", "B"):
        seq = [o for o, n in timed if n == name]
        assert seq == ["up", "solve", "down"] * (len(seq) // 3), seq
    assert [n for o, n in timed if o == "solve"] == ["A", "B", "A", "B", "A"]


def test_e2e_pipeline_reraises_a_side_thread_error():
    """An upload that fails on the side thread is raised on the main thread
    once the step's solve has returned (the side thread is joined first)."""
    import types

    import bench

    class Ev:
        def __init__(self, enable_timing=False):
            pass

        def record(self, s):
            pass

        def synchronize(self):
            pass

        def elapsed_time(self, other):
            return 1.0

    fake_torch = types.SimpleNamespace(cuda=types.SimpleNamespace(
        synchronize=lambda: None, ExternalStream=lambda p: p, Event=Ev))
    solves = []

    class FakeBatch:
        def __init__(self, name):
            self.name, self.stream = name, 0

        def solve(self, tol, max_iter):
            solves.append(self.name)

    uploads = []

    def upload(X):
        uploads.append(X.name)
        if len(uploads) > 3:  # the warm-up's two and the first timed one succeed
            raise RuntimeError("upload failed")

    with pytest.raises(RuntimeError, match="upload failed"):
        bench.e2e_pipelined(fake_torch, (FakeBatch("A"), FakeBatch("B")), upload, lambda X: None, 4)
    assert solves == ["A", "B", "A"]  # the step whose side thread failed still finished its solve
