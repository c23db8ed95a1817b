"""Host-side logic: input checks, synthetic inputs, batch sharding."""

import os
import warnings

import numpy as np
import pytest

from tests.conftest import golden
import torch.distributed as dist
import torch.multiprocessing as mp

import oracle
from pymatting_b200.shard import shard_sizes
from pymatting_b200.synthetic import batch_sizes, make_matting_problem
from pymatting_b200.util import sanity_check_image, trimap_split


def test_trimap_split_matches_oracle():
    rng = np.random.default_rng(0)
    t = rng.choice([0.0, 0.05, 0.5, 0.95, 1.0], size=(17, 23))
    for a, b in zip(trimap_split(t), oracle.trimap_split(t)):
        np.testing.assert_array_equal(a, b)
    fg, bg, known, unknown = trimap_split(t, flatten=False)
    assert fg.shape == (17, 23)


def test_trimap_split_errors_and_warnings():
    with pytest.raises(ValueError, match="background"):
        trimap_split(np.array([[1.0, 0.5]]))
    with pytest.raises(ValueError, match="foreground"):
        trimap_split(np.array([[0.0, 0.5]]))
    with warnings.catch_warnings(record=True) as w:
        warnings.simplefilter("always")
        trimap_split(np.array([[-0.5, 1.5]]))
        trimap_split(np.array([[0, 1]], dtype=np.int64))
    assert len(w) == 3


def test_sanity_check_image_warnings():
    with warnings.catch_warnings(record=True) as w:
        warnings.simplefilter("always")
        sanity_check_image((np.random.default_rng(0).standard_normal((8, 8, 2)) * 255)
                           .astype(np.int32))
    assert len(w) == 4


def test_synthetic_is_deterministic_and_calibrated():
    a = make_matting_problem(120, 160, 5, sigma=2.0, band=7, unknown_fraction=0.12)
    b = make_matting_problem(120, 160, 5, sigma=2.0, band=7, unknown_fraction=0.12)
    for x, y in zip(a[:3], b[:3]):
        np.testing.assert_array_equal(x, y)
    img, tri, alpha, frac = a
    assert img.shape == (120, 160, 3) and tri.shape == (120, 160)
    assert 0.0 <= img.min() and img.max() <= 1.0
    assert set(np.unique(tri)) <= {0.0, 0.5, 1.0}
    assert (tri == 1.0).any() and (tri == 0.0).any()
    assert abs(frac - np.mean(tri == 0.5)) < 1e-12


def test_batch_sizes():
    spec = batch_sizes(64, 1000)
    assert len(spec) == 64
    assert all(0.05 <= f <= 0.25 for _h, _w, f, _s in spec)
    assert spec == batch_sizes(64, 1000)


@pytest.mark.parametrize("world", [1, 2, 3, 8])
def test_shard_sizes_partition(world):
    sizes = [(h, w) for h, w, _f, _s in batch_sizes(64, 1000)]
    parts = shard_sizes(sizes, world)
    flat = sorted(k for p in parts for k in p)
    assert flat == list(range(64))
    loads = [sum(sizes[k][0] * sizes[k][1] for k in p) for p in parts]
    biggest = max(h * w for h, w in sizes)
    assert max(loads) - min(loads) <= biggest


def _gloo_worker(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    sizes = [(h, w) for h, w, _f, _s in batch_sizes(64, 1000)]
    mine = shard_sizes(sizes, world)[rank]
    gathered = [None] * world
    dist.all_gather_object(gathered, mine)
    if rank == 0:
        out.put(gathered)
    dist.barrier()
    dist.destroy_process_group()


def test_shard_ranks_agree_without_communication():
    """Each rank computes its shard alone; the union over ranks is the batch."""
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + (os.getpid() % 2000)
    procs = [ctx.Process(target=_gloo_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    gathered = q.get(timeout=120)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert sorted(k for part in gathered for k in part) == list(range(64))
    assert not set(gathered[0]) & set(gathered[1])


def _gather_worker(rank, world, port, out):
    """Shard the 64-image batch, 'solve' each image with a CPU stand-in
    (alpha = clipped trimap of a small synthetic image of that seed), gather
    the alphas and a statistics row per image to rank 0 over gloo."""
    import torch
    from pymatting_b200.shard import STAT_FIELDS, gather_images
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    spec = batch_sizes(64, 1000)
    sizes = [(h // 32, w // 32) for h, w, _f, _s in spec]
    parts = shard_sizes(sizes, world)

    def standin(k):
        h, w = sizes[k]
        _i, tri, _a, _f = make_matting_problem(h, w, spec[k][3], sigma=1.0, band=1,
                                               unknown_fraction=0.2)
        return torch.from_numpy(np.clip(tri, 0, 1)).reshape(-1)

    alphas = [standin(k) for k in parts[rank]]
    stats = [torch.tensor([float(k), 1.0, 1e-3, 1.0, float(rank)], dtype=torch.float64)
             for k in parts[rank]]
    cpu = torch.device("cpu")
    got = gather_images(alphas, sizes, parts, rank, world, cpu)
    got_st = gather_images(stats, [len(STAT_FIELDS)] * len(sizes), parts, rank, world, cpu)
    if rank == 0:
        ok = all(torch.equal(got[k], standin(k)) for k in range(len(sizes)))
        order = [int(s[0]) for s in got_st]
        owner = [int(s[4]) for s in got_st]
        out.put((ok, order, owner, [list(p) for p in parts]))
    else:
        assert got is None and got_st is None
    dist.barrier()
    dist.destroy_process_group()


def test_gather_to_rank0_in_batch_order():
    """The final gather of per-image alphas and statistics (gloo, 2 ranks):
    rank 0 receives every image once, in batch order, from the rank that
    owns it."""
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 31500 + (os.getpid() % 2000)
    procs = [ctx.Process(target=_gather_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    ok, order, owner, parts = q.get(timeout=180)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert ok
    assert order == list(range(64))
    for r, part in enumerate(parts):
        assert all(owner[k] == r for k in part)


def test_bench_starts_its_own_ranks():
    """bench.py --gpus 2 without a torch.distributed environment starts two
    ranks itself; its CPU plumbing check shards the batch and gathers it to
    rank 0, which prints the line."""
    import json
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    env = {k: v for k, v in os.environ.items()
           if k not in ("WORLD_SIZE", "RANK", "LOCAL_RANK", "MASTER_ADDR", "MASTER_PORT")}
    out = subprocess.run([sys.executable, os.path.join(root, "bench.py"), "--gpus", "2",
                          "--plumbing-check"], capture_output=True, text=True, timeout=300,
                         env=env, cwd=root)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [ln for ln in out.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    rec = json.loads(lines[0])
    assert rec["n_gpus"] == 2 and rec["images"] == 64 and rec["order_ok"]
    assert sum(rec["images_per_rank"]) == 64


def test_integration_rebinds_every_reexport():
    """The integration stub on PyMatting's own module layout
    (tests/golden/reference_layout.json, recorded from the imported
    reference): every module attribute bound to a replaced function — the
    defining module, the package re-exports under submodule names, and the
    names other modules imported — resolves to pymatting_b200 afterwards.
    Stand-in module objects carry the layout; no kernel is called."""
    import json
    import types
    import pymatting_b200 as b200
    from pymatting_b200 import integration
    with open(os.path.join(os.path.dirname(__file__), "golden", "reference_layout.json")) as f:
        layout = json.load(f)
    originals = {}

    def original(defmod, name):
        key = (defmod, name)
        if key not in originals:
            originals[key] = type(name, (), {}) if name[0].isupper() else (lambda *a: None)
        return originals[key]

    mods = {}
    for mname, attrs in layout.items():
        m = types.ModuleType(mname)
        for attr, (defmod, name) in attrs.items():
            setattr(m, attr, original(defmod, name))
        mods[mname] = m
    hot = {tuple(r) for r in integration.HOT_PATH}
    n_hot = sum(1 for attrs in layout.values() for v in attrs.values() if tuple(v) in hot)
    assert integration.install(include_next=False, modules=mods) == n_hot
    integration.uninstall()
    assert all(getattr(mods[m], a) is original(*v) for m, attrs in layout.items()
               for a, v in attrs.items())
    total = sum(len(a) for a in layout.values())
    assert integration.install(modules=mods) == total
    for mname, attrs in layout.items():
        for attr, (defmod, name) in attrs.items():
            assert getattr(mods[mname], attr) is getattr(b200, name), (mname, attr)
    # The bindings the reference's own call sites go through.
    assert mods["pymatting.laplacian"].cf_laplacian is b200.cf_laplacian
    assert mods["pymatting.preconditioner"].vcycle is b200.vcycle
    assert mods["pymatting"].make_linear_system is b200.make_linear_system
    ecf = mods["pymatting.alpha.estimate_alpha_cf"]
    assert ecf.cf_laplacian is b200.cf_laplacian and ecf.cg is b200.cg and ecf.ichol is b200.ichol
    integration.uninstall()


def _write_png(path, arr):
    from PIL import Image
    Image.fromarray(arr).save(path)


def test_image_file_helpers(tmp_path):
    """load_image / save_image / stack_images / blend (pymatting/util/util.py)
    on the reference test's own files (tests/golden/cutout_test.npz)."""
    import pymatting_b200 as pm
    g = golden("cutout_test.npz")
    p = str(tmp_path / "test.png")
    _write_png(p, g["test_u8"])
    img = pm.load_image(p)
    assert img.dtype == np.float64 and np.array_equal(img, g["test_u8"] / 255.0)
    rgb = pm.load_image(p, "RGB")
    assert rgb.shape == (32, 32, 3) and np.array_equal(rgb, g["test_u8"][:, :, :3] / 255.0)
    pa = str(tmp_path / "alpha.png")
    _write_png(pa, g["test_alpha_u8"])
    assert np.array_equal(pm.load_image(pa, "GRAY"), g["true_alpha"])
    half = pm.load_image(p, "RGB", 0.5, "box")
    assert half.shape == (16, 16, 3)
    out = str(tmp_path / "sub" / "out.png")
    pm.save_image(out, rgb)
    assert np.array_equal(pm.load_image(out), np.clip(rgb * 255, 0, 255).astype(np.uint8) / 255.0)
    st = pm.stack_images(rgb, g["true_alpha"])
    assert st.shape == (32, 32, 4) and np.array_equal(st[:, :, 3], g["true_alpha"])
    b = pm.blend(rgb, 1.0 - rgb, g["true_alpha"])
    a = g["true_alpha"][:, :, None]
    assert np.array_equal(b, a * rgb + (1 - a) * (1.0 - rgb))


def test_cutout_size_mismatch(tmp_path):
    import pymatting_b200 as pm
    g = golden("cutout_test.npz")
    p, t = str(tmp_path / "i.png"), str(tmp_path / "t.png")
    _write_png(p, g["test_u8"])
    _write_png(t, g["test_trimap_u8"][:16])
    with pytest.raises(ValueError):
        pm.cutout(p, t, str(tmp_path / "o.png"))


def test_foreground_level_plan_matches_oracle():
    """The host-side level sizes of estimate_foreground_ml (library, no GPU
    needed) equal the oracle's restatement of the reference's
    round(w0 ** (i / n)) schedule, including powers of two, strips and a
    1x1 image (ZeroDivisionError, as in the reference)."""
    import oracle
    from pymatting_b200.foreground import foreground_levels
    rng = np.random.default_rng(17)
    shapes = [(1, 2), (2, 1), (2, 2), (3, 1), (1, 1000), (31, 33), (32, 32), (64, 64), (1080, 1920),
              (2160, 3840), (4096, 4096), (4097, 3), (10000, 3), (65535, 2)]
    shapes += [tuple(int(v) for v in rng.integers(1, 5000, size=2)) for _ in range(200)]
    for h, w in shapes:
        if max(h, w) == 1:
            continue
        assert foreground_levels(h, w) == oracle.fg_levels(h, w), (h, w)
    with pytest.raises(ZeroDivisionError):
        foreground_levels(1, 1)
    with pytest.raises(ZeroDivisionError):
        oracle.fg_levels(1, 1)


def test_window_extent_prefixes_match_brute_force():
    """Row-pointer prefixes of the device Laplacians (host side): the
    clamped-window widths of uniform/rw and the shared-window widths of lbdm,
    against direct counts."""
    from pymatting_b200.laplacian import _lbdm_extents, _window_extents
    for n in (1, 2, 3, 5, 8, 17):
        for r in (1, 2, 3):
            brute = [len({min(max(v + d, 0), n - 1) for d in range(-r, r + 1)}) for v in range(n)]
            assert list(np.diff(_window_extents(n, r))) == brute, (n, r)
            if n > 2 * r:
                centres = range(r, n - r)
                brute = []
                for v in range(n):
                    cs = [c for c in centres if abs(c - v) <= r]
                    brute.append(len({q for c in cs for q in range(c - r, c + r + 1)}))
                assert list(np.diff(_lbdm_extents(n, r))) == brute, (n, r)


def test_laplacian_argument_errors():
    """Errors raised on the host before any device work, as in the reference."""
    import pymatting_b200 as pm
    img = np.zeros((6, 7, 3))
    with pytest.raises(ValueError):
        pm.knn_laplacian(img, kernel="gaussian")
    with pytest.raises(NotImplementedError):
        pm.lbdm_laplacian(img, radius=3)


def test_foreground_cf_neighbour_sets():
    import pymatting_b200 as pm
    with pytest.raises(NotImplementedError):
        pm.estimate_foreground_cf(np.zeros((4, 4, 3)), np.zeros((4, 4)), neighbors=[(1, 1)])


@pytest.mark.parametrize("workload", ["foreground", "hard320"])
def test_bench_reference_arm_line(workload):
    """bench.py --impl reference --workload foreground / hard320 runs the
    oracle on the host and prints one JSON line with the contract's keys."""
    import json
    import subprocess
    import sys
    import os
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    out = subprocess.run([sys.executable, os.path.join(root, "bench.py"), "--impl", "reference",
                          "--workload", workload, "--steps", "1", "--warmup", "0"],
                         capture_output=True, text=True, timeout=600, cwd=root)
    assert out.returncode == 0, out.stderr[-2000:]
    line = json.loads(out.stdout.strip().splitlines()[-1])
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step",
                "higher_is_better", "impl", "cpu_baseline", "e2e", "config"):
        assert key in line, key
    assert line["impl"] == "reference" and line["value"] > 0
    assert line["e2e"]["h2d_bytes_per_step"] == 0
