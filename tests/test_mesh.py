"""Synthetic workload generators: sizes, tensor node order, seeds."""
import numpy as np

from gpu_fem_b200 import mesh as M


def _normals_positive(mesh):
    X = mesh.xpts[mesh.conn]
    n = np.cross(X[:, 1] - X[:, 0], X[:, 2] - X[:, 0])
    return (np.linalg.norm(n, axis=1) > 0).all()


def test_config1_sizes():
    m = M.plate_config1()
    assert (m.num_nodes, m.num_elements, m.num_dof) == (121, 100, 726)
    assert len(m.bcs) == 6 * 40
    # 81 interior nodes carry h^2 p = 0.01 m^2 * 1 kPa each
    assert abs(m.loads.sum() - 810.0) < 1e-9


def test_config2_sizes_and_jitter():
    m = M.plate_config2()
    assert (m.num_nodes, m.num_elements) == (80601, 80000)
    h = 0.005
    ix = np.rint(m.xpts[:, 0] / h)
    assert np.abs(m.xpts[:, 0] - ix * h).max() <= 0.1 * h + 1e-15
    assert m.thick.min() >= 0.004 * 0.75 - 1e-12 and m.thick.max() <= 0.004 * 1.25 + 1e-12
    assert _normals_positive(m)
    # corners fixed, deterministic
    m2 = M.plate_config2()
    assert np.array_equal(m.xpts, m2.xpts)


def test_box_small_topology():
    b = M.box(nx=18, ny=6, nz=4, nribs=4)
    assert b.num_elements == 2 * 18 * 6 + 2 * 18 * 4 + 4 * 6 * 4
    assert _normals_positive(b)
    assert abs(b.loads.sum() - 1e4) < 1e-6


def test_batch_config4_seeded():
    probs = M.batch_config4()
    assert len(probs) == 64
    sizes = [p.num_elements for p in probs]
    assert min(sizes) >= 16 * 16 and max(sizes) <= 256 * 256
    assert sizes == [p.num_elements for p in M.batch_config4()]


def test_step_cost_model_prefers_what_the_kernels_reward():
    """The autotuner's step model: a longer factor row costs more in the
    factorization, more levels cost in every GMRES step, and levels big
    enough for two CTAs are cheaper per block."""
    from gpu_fem_b200.batch import step_cost_us
    n = 20000
    short = step_cost_us(n, {"levels_L": 1000, "levels_U": 1000, "nnzb": 20 * n}, 50)
    long_rows = step_cost_us(n, {"levels_L": 1000, "levels_U": 1000, "nnzb": 40 * n}, 50)
    assert long_rows > short
    deeper = step_cost_us(n, {"levels_L": 2000, "levels_U": 2000, "nnzb": 20 * n}, 50)
    assert deeper > short
    more_its = step_cost_us(n, {"levels_L": 1000, "levels_U": 1000, "nnzb": 20 * n}, 100)
    assert more_its > short
    # per level: one CTA for small levels, two for large ones (cheaper per block)
    one = step_cost_us(n, {"levels_L": 2000, "levels_U": 2000, "nnzb": n + 2 * 2000 * 190}, 10)
    two = step_cost_us(n, {"levels_L": 2000, "levels_U": 2000, "nnzb": n + 2 * 2000 * 400}, 10)
    assert two < 2 * one


def test_batch_objective_lowers_fill_of_early_converging_problems():
    """In a batch, GMRES runs as many steps as the slowest problem needs and
    each launch lasts as long as its longest level chain: a problem that
    converges early at high fill is better off at a lower fill with more
    (but still fewer than the batch's) steps."""
    from gpu_fem_b200.batch import batch_cost_us, choose_batch_fills
    slow = [(5, 100, 1000.0, 500.0)]                       # (k, steps, factor us, sweep us)
    fast = [(8, 10, 5000.0, 2000.0), (3, 60, 500.0, 600.0)]
    # 1000 + 60 x (600 + 150) + 40 x (500 + 150)
    assert batch_cost_us([(100, 1000.0, 500.0), (60, 500.0, 600.0)]) == 72000.0
    # 5000 + 10 x (2000 + 150) + 90 x (500 + 150)
    assert batch_cost_us([(100, 1000.0, 500.0), (10, 5000.0, 2000.0)]) == 85000.0
    fills, cost = choose_batch_fills([slow, fast])
    assert fills == [5, 3] and cost == 72000.0
    # alone, the fast problem's own cheapest candidate is the high fill
    from gpu_fem_b200.batch import STEP_OVERHEAD_US
    own = min(fast, key=lambda t: t[2] + t[1] * (t[3] + STEP_OVERHEAD_US))
    assert own[0] == 8


def test_shared_factor_costs_charge_the_sm_share():
    """In a batch the factorization's CTAs are shared out by block updates:
    a heavy candidate of one problem among heavy others gets fewer SMs and
    costs more than alone; without the others it costs what it costs alone."""
    from gpu_fem_b200.batch import factor_cost_us, shared_factor_costs
    n = 20000
    inf = {"levels_L": 2000, "levels_U": 2000, "nnzb": 30 * n, "ordering": "natural"}
    cand = (12, 20, factor_cost_us(n, inf), 500.0, (n, inf))
    alone = shared_factor_costs([[cand]], [12])[0][0][2]
    assert abs(alone - factor_cost_us(n, inf, warps=8 * 128)) < 1e-9
    crowd = shared_factor_costs([[cand]] * 8, [12] * 8)[0][0][2]
    assert crowd > alone
    assert shared_factor_costs([[cand]], None)[0][0] == cand[:4]
