"""GPU stream frames (sss_stream_sample / sss_stream_minmax) against the
golden frames of the reference's own build_frame: the box, the culled and
thinned index lists and the u16 coordinates of both samples, bit for bit,
in linear and in log zoom (f32 hypot and log1p computed as the C library
does, which NumPy calls for them when its SIMD dispatch is off)."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

SCENES = ["wolken", "massenwolke", "autobox_log", "klein_tot"]


@pytest.mark.parametrize("scene", SCENES)
def test_frames_match_reference(load_golden, scene):
    from solarsystemsimulator_b200.stream import StreamFrames
    g = load_golden(f"server_frame_{scene}.npz")
    log_zoom = bool(g["log_zoom"])
    sf = StreamFrames(g["is_ast"], g["injected"])
    sf.kill_t = torch.as_tensor(g["kill_t"]).cuda()
    x0, y0 = torch.as_tensor(g["x0"]).cuda(), torch.as_tensor(g["y0"]).cuda()
    box = sf.box(x0, y0, tuple(g["view"]), log_zoom)
    assert box == tuple(float(v) for v in g["box"])
    for k in range(2):
        t_i = float(g["t0"]) + (k + 1) * float(g["raster_days"])
        x, y = torch.as_tensor(g[f"x{k}"]).cuda(), torch.as_tensor(g[f"y{k}"]).cuda()
        sel, qx, qy = (t.cpu().numpy() for t in sf.sample(x, y, t_i, float(g["raster_days"]), box, log_zoom,
                                                          int(g["budget"])))
        sel = sel.view(np.uint32)
        qx = qx.view(np.uint16)
        qy = qy.view(np.uint16)
        assert np.array_equal(sel, g[f"sel{k}"])
        assert np.array_equal(qx, g[f"qx{k}"]) and np.array_equal(qy, g[f"qy{k}"])


def _scene(n_mass, n_ast, n_inj, seed, spread=1.0):
    rng = np.random.default_rng(seed)
    n = n_mass + n_ast + n_inj
    x = np.zeros(n)
    y = np.zeros(n)
    x[:n_mass] = rng.uniform(-5, 5, n_mass)
    y[:n_mass] = rng.uniform(-5, 5, n_mass)
    cen = rng.uniform(-3, 3, (8, 2))
    lab = rng.integers(0, 8, n_ast + n_inj)
    sig = 10 ** rng.uniform(-2.5, -0.3, 8) * spread
    x[n_mass:] = cen[lab, 0] + rng.normal(0, 1, n_ast + n_inj) * sig[lab]
    y[n_mass:] = cen[lab, 1] + rng.normal(0, 1, n_ast + n_inj) * sig[lab]
    is_ast = np.zeros(n, bool)
    is_ast[n_mass:] = True
    inj = np.zeros(n, bool)
    inj[n_mass + n_ast:] = True
    kill_t = np.full(n, np.inf)
    dead = rng.choice(n, n // 50, replace=False)
    kill_t[dead] = rng.uniform(-1, 1, len(dead))
    return x.astype(np.float32), y.astype(np.float32), is_ast, inj, kill_t


# (masses, system asteroids, injected, view, budget): the film's full LOD
# budget over 600k bodies, the self-gravity cloud branch, a budget below
# the masses (masses only) and a box that holds nobody
LARGE = {
    "asteroids_600k": (20, 500_000, 100_000, (0.0, 0.0, 2.0, 2.0), 120_000),
    "mass_cloud": (40_000, 200_000, 0, (0.5, 0.0, 3.0, 3.0), 30_000),
    "masses_only": (150, 50_000, 0, (0.0, 0.0, 4.0, 4.0), 100),
    "empty_box": (10, 10_000, 1000, (400.0, 400.0, 1.0, 1.0), 1000),
}


@pytest.mark.parametrize("name", list(LARGE))
def test_large_samples_match_oracle(name):
    """Linear display coordinates at film sizes: bit-exact against the oracle."""
    from oracle import frames as ofr
    from solarsystemsimulator_b200.stream import StreamFrames
    nm, na, ni, view, budget = LARGE[name]
    x, y, a, inj, kill_t = _scene(nm, na, ni, seed=len(name))
    sf = StreamFrames(a, inj)
    sf.kill_t = torch.as_tensor(kill_t).cuda()
    xd, yd = torch.as_tensor(x).cuda(), torch.as_tensor(y).cuda()
    box = sf.box(xd, yd, view, False)
    assert box == ofr.make_box(x, y, view)
    t_i = 0.5
    sel, qx, qy = (t.cpu().numpy() for t in sf.sample(xd, yd, t_i, 0.5, box, False, budget))
    rs, rx, ry = ofr.sample_frame(x, y, kill_t > 0.0, a, inj, box, False, budget)
    assert np.array_equal(sel.view(np.uint32), rs)
    assert np.array_equal(qx.view(np.uint16), rx) and np.array_equal(qy.view(np.uint16), ry)
    if name == "empty_box":
        assert len(rs) == 0
    else:
        assert 0 < len(rs) <= max(budget, nm) * 1.05


def test_autobox_matches_oracle_log_zoom():
    """Automatic box (no view yet) and the log zoom at 300k bodies."""
    from oracle import frames as ofr
    from solarsystemsimulator_b200.stream import StreamFrames
    x, y, a, inj, kill_t = _scene(9, 300_000, 0, seed=3, spread=3.0)
    sf = StreamFrames(a, inj)
    xd, yd = torch.as_tensor(x).cuda(), torch.as_tensor(y).cuda()
    box_lin = sf.box(xd, yd, (0, 0, -1, -1), False)
    assert box_lin == ofr.make_box(x, y, (0, 0, -1, -1))
    qx0, qy0 = ofr.display_coords(x, y, True)
    ref_box = ofr.make_box(qx0, qy0, (0, 0, -1, -1))
    box = sf.box(xd, yd, (0, 0, -1, -1), True)
    assert box == ref_box
    sel, qx, qy = (t.cpu().numpy() for t in sf.sample(xd, yd, 0.5, 0.5, box, True, 60_000))
    rs, rx, ry = ofr.sample_frame(x, y, np.ones(len(x), bool), a, inj, ref_box, True, 60_000)
    assert np.array_equal(sel.view(np.uint32), rs)
    assert np.array_equal(qx.view(np.uint16), rx) and np.array_equal(qy.view(np.uint16), ry)


def test_log_zoom_display_coordinates_bit_exact():
    """The display scale at every radius the film can show (1e-9 to 1e4 AU,
    log-uniform, plus the branch points of the log1p reduction) equals the
    oracle's bit for bit."""
    from oracle import frames as ofr
    from solarsystemsimulator_b200.stream import StreamFrames
    rng = np.random.default_rng(21)
    n = 2_000_000
    r = np.exp(rng.uniform(np.log(1e-9), np.log(1e4), n))
    th = rng.uniform(0, 2 * np.pi, n)
    x = (r * np.cos(th)).astype(np.float32)
    y = (r * np.sin(th)).astype(np.float32)
    edge = np.array([0x3ED413D5, 0x3ED413D6, 0x3ED413D7, 0x3ED413DA, 0x3504F3 | 0x3F800000, 0x31000000,
                     0x30FFFFFF, 0x5A000000, 0x3F800000], np.int32).view(np.float32)
    x = np.concatenate([x, edge, np.zeros(3, np.float32)])
    y = np.concatenate([y, np.zeros(len(edge), np.float32), np.array([0.0, 1e-9, 2e-9], np.float32)])
    a = np.ones(len(x), bool)
    sf = StreamFrames(a, np.zeros(len(x), bool))
    qx, qy = sf.display(torch.as_tensor(x).cuda(), torch.as_tensor(y).cuda())
    rx, ry = ofr.display_coords(x, y, True)
    assert np.array_equal(qx.cpu().numpy().view(np.int32), rx.view(np.int32))
    assert np.array_equal(qy.cpu().numpy().view(np.int32), ry.view(np.int32))


def test_kill_times():
    from solarsystemsimulator_b200.stream import StreamFrames
    x, y, a, inj, _ = _scene(5, 2000, 0, seed=1)
    sf = StreamFrames(a, inj)
    sf.kill([7, 9, 11], 0.25)
    sf.kill([9], 1.0)                     # a later kill does not revive an earlier one
    xd, yd = torch.as_tensor(x).cuda(), torch.as_tensor(y).cuda()
    box = (-100.0, -100.0, 200.0, 200.0)
    sel = sf.sample(xd, yd, 0.5, 0.5, box, False, 10**6)[0].cpu().numpy()
    assert len(sel) == len(x) and 7 in sel                  # t_cut 0.0 < 0.25
    sel = sf.sample(xd, yd, 1.0, 0.5, box, False, 10**6)[0].cpu().numpy()
    assert len(sel) == len(x) - 3 and not {7, 9, 11} & set(sel.tolist())


@pytest.mark.parametrize("scene", SCENES)
def test_batch_equals_single_samples(load_golden, scene):
    """sample_batch (both samples of the golden frame in one call) gives the
    golden frames and the single-sample results."""
    from solarsystemsimulator_b200.stream import StreamFrames
    g = load_golden(f"server_frame_{scene}.npz")
    log_zoom = bool(g["log_zoom"])
    sf = StreamFrames(g["is_ast"], g["injected"])
    sf.kill_t = torch.as_tensor(g["kill_t"]).cuda()
    box = tuple(float(v) for v in g["box"])
    rd = float(g["raster_days"])
    xs = [torch.as_tensor(g[f"x{k}"]).cuda() for k in range(2)]
    ys = [torch.as_tensor(g[f"y{k}"]).cuda() for k in range(2)]
    ts = [float(g["t0"]) + (k + 1) * rd for k in range(2)]
    batch = [tuple(t.cpu().numpy() for t in r) for r in sf.sample_batch(xs, ys, ts, rd, box, log_zoom, int(g["budget"]))]
    for k in range(2):
        single = tuple(t.cpu().numpy() for t in sf.sample(xs[k], ys[k], ts[k], rd, box, log_zoom, int(g["budget"])))
        for a, b in zip(batch[k], single):
            assert np.array_equal(a, b)
        if not log_zoom:
            assert np.array_equal(batch[k][0].view(np.uint32), g[f"sel{k}"])
            assert np.array_equal(batch[k][1].view(np.uint16), g[f"qx{k}"])


def test_batch_of_twenty():
    """A batch longer than the stack buffer of control blocks (20 samples of
    110,000 bodies moving between samples, LOD active): every sample as its
    single-sample call."""
    from solarsystemsimulator_b200.stream import StreamFrames
    x, y, a, inj, kill_t = _scene(20, 100_000, 10_000, seed=4)
    sf = StreamFrames(a, inj)
    sf.kill_t = torch.as_tensor(kill_t).cuda()
    rng = np.random.default_rng(5)
    xs, ys = [], []
    for k in range(20):
        xs.append(torch.as_tensor((x + rng.normal(0, 1e-3, len(x))).astype(np.float32)).cuda())
        ys.append(torch.as_tensor((y + rng.normal(0, 1e-3, len(y))).astype(np.float32)).cuda())
    ts = [0.1 * (k + 1) for k in range(20)]
    box = sf.box(xs[0], ys[0], (0.0, 0.0, 2.0, 2.0), False)
    batch = [tuple(t.cpu().numpy() for t in r) for r in sf.sample_batch(xs, ys, ts, 0.1, box, False, 20_000)]
    for k in range(20):
        single = [t.cpu().numpy() for t in sf.sample(xs[k], ys[k], ts[k], 0.1, box, False, 20_000)]
        assert all(np.array_equal(p, q) for p, q in zip(batch[k], single))
        assert 0 < len(single[0]) <= 25_000


def test_many_distinct_cell_counts_take_the_exact_rounds():
    """4,200 distinct cell counts (cell i of the box holds i + 1 bodies,
    8,822,100 asteroids): more than the count histogram holds, so the
    bisection runs entirely in the exact pairwise rounds; bit-exact against
    the oracle."""
    from oracle import frames as ofr
    from solarsystemsimulator_b200.stream import StreamFrames
    k, cells = 512, 4200
    reps = np.arange(1, cells + 1)
    cid = np.repeat(np.arange(cells), reps)
    rng = np.random.default_rng(17)
    x = ((cid % k + 0.5 + rng.uniform(-0.3, 0.3, len(cid))) / k).astype(np.float32)
    y = ((cid // k + 0.5 + rng.uniform(-0.3, 0.3, len(cid))) / k).astype(np.float32)
    n = len(x)
    a = np.ones(n, bool)
    inj = np.zeros(n, bool)
    view = (0.5, 0.5, 0.25, 0.25)                     # box (0, 0, 1, 1): one LOD cell per grid cell
    box = ofr.make_box(x, y, view)
    sf = StreamFrames(a, inj)
    xd, yd = torch.as_tensor(x).cuda(), torch.as_tensor(y).cuda()
    assert sf.box(xd, yd, view, False) == box
    sel, qx, qy = (t.cpu().numpy() for t in sf.sample(xd, yd, 0.5, 0.5, box, False, 120_000))
    rs, rx, ry = ofr.sample_frame(x, y, np.ones(n, bool), a, inj, box, False, 120_000)
    assert np.array_equal(sel.view(np.uint32), rs)
    assert np.array_equal(qx.view(np.uint16), rx) and np.array_equal(qy.view(np.uint16), ry)
    assert 100_000 < len(rs) < 140_000


# cell counts that reach each path of the count histogram: counts on both
# sides of the direct table's end (4096), up to 512 larger counts (ranked)
# and more (bitonic network), and more than 1024 distinct counts (prefix
# sums in global memory)
HIST_CASES = {
    "direct_1500": np.arange(1, 1501),
    "across_4096": np.concatenate([np.arange(1, 1001), np.arange(4000, 4201)]),
    "ranked_300": np.concatenate([np.arange(1, 200), 4096 + 7 * np.arange(300)]),
    "bitonic_600": np.concatenate([np.arange(1, 100), 4096 + np.arange(600)]),
}


@pytest.mark.parametrize("name", list(HIST_CASES))
def test_count_histogram_paths(name):
    """Cell j of a shuffled set of LOD cells holds counts[j] asteroids:
    bit-exact against the oracle, with the LOD budget thinning them."""
    from oracle import frames as ofr
    from solarsystemsimulator_b200.stream import StreamFrames
    k = 512
    counts = HIST_CASES[name]
    rng = np.random.default_rng(len(name))
    cells = rng.choice(k * k, len(counts), replace=False)
    cid = np.repeat(cells, counts)
    x = ((cid % k + 0.5 + rng.uniform(-0.3, 0.3, len(cid))) / k).astype(np.float32)
    y = ((cid // k + 0.5 + rng.uniform(-0.3, 0.3, len(cid))) / k).astype(np.float32)
    n = len(x)
    a = np.ones(n, bool)
    inj = np.zeros(n, bool)
    view = (0.5, 0.5, 0.25, 0.25)                     # box (0, 0, 1, 1): one LOD cell per grid cell
    box = ofr.make_box(x, y, view)
    sf = StreamFrames(a, inj)
    xd, yd = torch.as_tensor(x).cuda(), torch.as_tensor(y).cuda()
    assert sf.box(xd, yd, view, False) == box
    sel, qx, qy = (t.cpu().numpy() for t in sf.sample(xd, yd, 0.5, 0.5, box, False, 120_000))
    rs, rx, ry = ofr.sample_frame(x, y, np.ones(n, bool), a, inj, box, False, 120_000)
    assert np.array_equal(sel.view(np.uint32), rs)
    assert np.array_equal(qx.view(np.uint16), rx) and np.array_equal(qy.view(np.uint16), ry)
    assert 80_000 < len(rs) <= 120_000
