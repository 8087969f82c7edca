"""GPU parity of every FAC level operator and of the whole solve against the
CPU oracle, through the C ABI.

Bars: ghost fills are bit-exact; smoothing, residual, flux, restriction,
prolongation and the converged solution match to 1e-12 relative (the FP64
kernels use the reference's operation order with FMA contraction off, so in
practice they are bit-exact too); norms to 1e-13 relative.
"""
import numpy as np
import pytest

from samrai_b200 import configs, fac
from oracle.oracle import C, E, F, Oracle, R, TR, U, W, SD

pytestmark = pytest.mark.gpu

REL = 1e-12


def rel_err(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    scale = max(np.abs(b).max(), 1e-300)
    return float(np.abs(a - b).max() / scale)


def pair(prob, params=None):
    o = Oracle(prob, params=params)
    g = fac.FacContext([prob], params=params)
    return o, g


def randomize(prob, o, g, rng, fields=(U, E, R, F, TR)):
    for ln in range(prob.nlev):
        for fid in fields:
            v = rng.standard_normal(o.size(fid, ln))
            o.set(fid, ln, v)
            g.upload(fid, 0, ln, v)


CONFIGS = [configs.config1, configs.config3, configs.small_3d]


@pytest.mark.parametrize("mk", CONFIGS + [configs.config2])
@pytest.mark.parametrize("homogeneous", [0, 1])
def test_ghost_fill_bit_exact(mk, homogeneous, require_gpu):
    p = mk()
    o, g = pair(p)
    randomize(p, o, g, np.random.default_rng(1))
    for ln in range(p.nlev):
        for with_coarse in ([0, 1] if ln > 0 else [0]):
            o.ghost_fill(U, ln, with_coarse, homogeneous)
            g.ghost_fill(U, ln, with_coarse, homogeneous)
            assert np.array_equal(g.download(U, 0, ln), o.get(U, ln)), (ln, with_coarse)


@pytest.mark.parametrize("mk", CONFIGS)
def test_smooth(mk, require_gpu):
    p = mk()
    o, g = pair(p)
    randomize(p, o, g, np.random.default_rng(2))
    for ln in range(p.nlev):
        o.smooth(E, R, ln, 2, -1.0)
        g.smooth(E, R, ln, 2, -1.0)
        assert rel_err(g.download(E, 0, ln), o.get(E, ln)) <= REL
        assert np.array_equal(g.download(E, 0, ln), o.get(E, ln))


@pytest.mark.parametrize("mk", [configs.config1, configs.small_3d])
def test_coarse_solve_sweep_count(mk, require_gpu):
    p = mk()
    o, g = pair(p, params=dict(coarse_tol=1e-3, coarse_max_it=200))
    randomize(p, o, g, np.random.default_rng(3), fields=(E, R))
    n_o, _ = o.smooth(E, R, 0, 200, 1e-3)
    n_g = g.smooth(E, R, 0, 200, 1e-3)
    assert int(n_g[0]) == n_o
    assert rel_err(g.download(E, 0, 0), o.get(E, 0)) <= REL


@pytest.mark.parametrize("mk", CONFIGS)
@pytest.mark.parametrize("error_eq", [0, 1])
def test_composite_residual(mk, error_eq, require_gpu):
    p = mk()
    o, g = pair(p)
    randomize(p, o, g, np.random.default_rng(4))
    for ln in range(p.nlev - 1, -1, -1):
        o.comp_residual(R, U, F, ln, error_eq)
        g.comp_residual(R, U, F, ln, error_eq)
        assert rel_err(g.download(R, 0, ln), o.get(R, ln)) <= REL, ln
        assert rel_err(g.download_flux(0, ln), o.get_side(1, ln)) <= REL, ln
        if ln > 0:
            assert rel_err(g.download_oside(0, ln), o.get_oside(ln)) <= REL, ln
        assert np.array_equal(g.download(U, 0, ln), o.get(U, ln))


@pytest.mark.parametrize("mk", CONFIGS)
def test_restrict_and_prolong(mk, require_gpu):
    p = mk()
    o, g = pair(p)
    randomize(p, o, g, np.random.default_rng(5))
    for ln in range(p.nlev - 2, -1, -1):
        o.restrict(TR, R, ln)
        g.restrict(TR, R, ln)
        assert rel_err(g.download(R, 0, ln), o.get(R, ln)) <= REL
        o.restrict_solution(U, ln)
        g.restrict_solution(U, ln)
        assert rel_err(g.download(U, 0, ln), o.get(U, ln)) <= REL
    for ln in range(1, p.nlev):
        o.prolong_correct(E, E, ln)
        g.prolong_correct(E, E, ln)
        assert rel_err(g.download(E, 0, ln), o.get(E, ln)) <= REL


@pytest.mark.parametrize("mk", CONFIGS)
def test_rms_norm(mk, require_gpu):
    p = mk()
    o, g = pair(p)
    randomize(p, o, g, np.random.default_rng(6), fields=(R,))
    o.compute_weights()
    g.compute_weights()
    for ln in range(p.nlev):
        assert np.array_equal(g.download(W, 0, ln), o.get(W, ln))
    assert abs(g.rms_norm(R)[0] - o.rms_norm(R)) <= 1e-13 * o.rms_norm(R)


def _solution_check(p, o, g, prob_index=0):
    for ln in range(p.nlev):
        assert rel_err(g.download(U, prob_index, ln), o.get(U, ln)) <= REL, ln


def test_full_solve_config1(require_gpu):
    p = configs.config1()
    prm = dict(coarse_tol=1e-10)
    o, g = pair(p, prm)
    ok_o, it_o, res_o, hist_o = o.solve()
    conv, its, res = g.solve()
    assert ok_o and conv[0]
    assert its[0] == it_o
    hist_g = g.residual_history(0)
    assert len(hist_g) == len(hist_o)
    assert rel_err(hist_g, hist_o) <= 1e-11
    _solution_check(p, o, g)
    assert np.array_equal(g.coarse_sweeps(), [o.coarse_sweeps()])


def test_full_solve_small_3d(require_gpu):
    p = configs.small_3d()
    prm = dict(coarse_tol=1e-10, max_cycles=6)
    o, g = pair(p, prm)
    o.solve()
    g.solve()
    assert len(g.residual_history(0)) == 7
    _solution_check(p, o, g)


def test_full_solve_varcoef_config3(require_gpu):
    p = configs.config3()
    prm = dict(coarse_tol=1e-10, max_cycles=8)
    o, g = pair(p, prm)
    ok_o, it_o, res_o, hist_o = o.solve()
    conv, its, res = g.solve()
    assert its[0] == it_o
    assert rel_err(g.residual_history(0), hist_o) <= 1e-11
    _solution_check(p, o, g)


def test_batched_problems_match_individual_oracles(require_gpu):
    probs = [configs.small_3d(seed=s) for s in (11, 12, 13)]
    prm = dict(coarse_tol=1e-10, max_cycles=4)
    g = fac.FacContext(probs, params=prm)
    g.solve()
    for i, p in enumerate(probs):
        o = Oracle(p, params=prm)
        o.solve()
        _solution_check(p, o, g, prob_index=i)


def test_config2_one_cycle(require_gpu):
    p = configs.config2()
    prm = dict(coarse_tol=1e-10, coarse_max_it=10, max_cycles=1)
    o, g = pair(p, prm)
    o.solve()
    g.solve()
    _solution_check(p, o, g)


def test_coarsest_one_launch_solve_matches_oracle(require_gpu):
    """Smoothing to a tolerance on a coarsest level with one patch per problem
    runs every sweep in one launch (one block per problem, the sweep check
    inside); per problem the sweep count and the result must equal the
    oracle's, for problems that stop after different sweep counts."""
    probs = [configs.extend_hierarchy(configs.small_3d(seed=s), k=2) for s in (71, 72, 73)]
    prm = dict(coarse_tol=1e-3, coarse_max_it=200)
    g = fac.FacContext(probs, params=prm)
    oracles = [Oracle(p, params=prm) for p in probs]
    rng = np.random.default_rng(74)
    for i, o in enumerate(oracles):
        for fid in (E, R):
            v = rng.standard_normal(o.size(fid, 0)) * (1.0 + 3.0 * i)
            o.set(fid, 0, v)
            g.upload(fid, i, 0, v)
    n_g = g.smooth(E, R, 0, 200, 1e-3)
    for i, o in enumerate(oracles):
        n_o, _ = o.smooth(E, R, 0, 200, 1e-3)
        assert int(n_g[i]) == n_o
        assert np.array_equal(g.download(E, i, 0), o.get(E, 0))
    g.close()


def test_mg_extended_hierarchy_matches_oracle(require_gpu):
    """The fast variant (hierarchy extended by fully covered coarser levels)
    against the oracle run on the same extended hierarchy, and its converged
    solution against the plain solve's."""
    p = configs.config3()
    x = configs.extend_hierarchy(p)
    prm = dict(coarse_tol=1e-300, coarse_max_it=20)
    o = Oracle(x, params=prm)
    g = fac.FacContext([x], params=prm)
    ok_o, it_o, res_o, hist_o = o.solve()
    conv, its, res = g.solve()
    assert ok_o and conv[0] and its[0] == it_o
    _solution_check(x, o, g)
    op = Oracle(p, params=dict(coarse_tol=1e-10))
    assert op.solve()[0]
    k = x.virtual_levels
    num = den = 0.0
    for ln in range(p.nlev):
        a = g.download(U, 0, ln + k)
        b = op.get(U, ln)
        num += float(np.sum((a - b) ** 2))
        den += float(np.sum(b ** 2))
    assert (num / den) ** 0.5 <= 1e-9


def test_no_presmoothing_matches_oracle(require_gpu):
    """Without pre-smoothing the cycle restricts f instead of forming the
    residual of the zero error (the same bits); the oracle forms it.  FP64
    stationary solve on the extended hierarchy: the same cycle count and
    residual history, the same solution."""
    p = configs.extend_hierarchy(configs.config3())
    prm = dict(coarse_tol=1e-300, coarse_max_it=40, pre_sweeps=0, post_sweeps=3)
    o = Oracle(p, params=prm)
    g = fac.FacContext([p], params=prm)
    ok_o, it_o, res_o, hist_o = o.solve()
    conv, its, res = g.solve()
    assert ok_o and conv[0] and its[0] == it_o
    assert rel_err(g.residual_history(0), hist_o) <= 1e-11
    _solution_check(p, o, g)
    g.close()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_no_presmoothing_fgmres_matches_oracle_solution(precision, require_gpu):
    """FGMRES with the cycle without pre-smoothing, both precisions: the
    solution of the oracle's converged plain solve."""
    p = configs.config3()
    x = configs.extend_hierarchy(p)
    prm = dict(coarse_tol=1e-300, coarse_max_it=40, pre_sweeps=0, post_sweeps=3,
               relative_residual_tol=1e-12, max_cycles=60)
    g = fac.FacContext([x], params=prm, precision=precision)
    g.set_krylov(20)
    conv, its, res = g.solve()
    assert conv[0]
    k = x.virtual_levels
    uk = [g.download(U, 0, ln + k) for ln in range(p.nlev)]
    g.close()
    op = Oracle(p, params=dict(coarse_tol=1e-12, relative_residual_tol=1e-12))
    assert op.solve()[0]
    assert _rel_l2(uk, [op.get(U, ln) for ln in range(p.nlev)]) <= 1e-9


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_graph_replay_matches_eager(precision, require_gpu):
    """fac_solve replays one captured CUDA graph per cycle; the eager launch
    sequence must give bit-identical results."""
    probs = [configs.extend_hierarchy(configs.small_3d(seed=s), k=2) for s in (31, 32)]
    prm = dict(coarse_tol=1e-300, coarse_max_it=20)
    out = []
    for graph in (True, False):
        g = fac.FacContext(probs, params=prm, precision=precision)
        g.set_graph(graph)
        conv, its, res = g.solve()
        out.append((its.copy(), [g.download(U, i, ln) for i in range(2)
                                 for ln in range(probs[0].nlev)]))
        g.close()
    assert np.array_equal(out[0][0], out[1][0])
    for a, b in zip(out[0][1], out[1][1]):
        assert np.array_equal(a, b)


def _fused_levels_2d(probs):
    """Levels whose patches all start on the same parity of lo0+lo1 (the
    condition under which the fused colour pass runs in 2-D)."""
    out = []
    for ln in range(probs[0].nlev):
        par = {int(b[0] + b[1]) % 2 for p in probs for b in p.levels[ln].boxes}
        if len(par) == 1:
            out.append(ln)
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("case", ["config1", "small_3d_mg", "config2"])
def test_fused_and_staged_colour_passes_match_filled(case, precision, require_gpu):
    """Colour passes that read across patch faces directly must give the same
    bits as passes that read ghost cells filled before each pass, including
    the ghost values left after the solve."""
    if case == "config1":
        probs = [configs.config1()]
        assert len(_fused_levels_2d(probs)) >= 1
    elif case == "config2":
        probs = [configs.config2()]
        assert _fused_levels_2d(probs) == list(range(probs[0].nlev))
    else:
        probs = [configs.extend_hierarchy(configs.small_3d(seed=s), k=2) for s in (41, 42)]
    prm = dict(coarse_tol=1e-300, coarse_max_it=20, max_cycles=2 if case == "config2" else 6)
    out = []
    # fused passes on staged shared-memory units (default stages; three and
    # four stages of small units, so that patches are cut into several
    # units), fused passes reading HBM, and passes between ghost fills
    for fused, staged, depth, budget in ((True, True, None, None), (True, True, 3, 8192),
                                         (True, True, 4, 4096), (True, False, None, None),
                                         (False, False, None, None)):
        g = fac.FacContext(probs, params=prm, precision=precision)
        g.set_fused(fused)
        g.set_staged(staged)
        if depth:
            g.set_stage_depth(depth)
            g.set_stage_budget(budget)
        conv, its, res = g.solve()
        fields = [g.download(U, i, ln) for i in range(len(probs)) for ln in range(probs[0].nlev)]
        g.smooth(E, R, probs[0].nlev - 1, 3)
        fields += [g.download(E, i, ln) for i in range(len(probs)) for ln in range(probs[0].nlev)]
        out.append((its.copy(), res.copy(), fields))
        g.close()
    for other in out[1:]:
        assert np.array_equal(out[0][0], other[0])
        assert np.array_equal(out[0][1], other[1])
        for a, b in zip(out[0][2], other[2]):
            assert np.array_equal(a, b)


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("case", ["config1", "small_3d_mg", "config3"])
def test_fused_residual_matches_flux_arrays(case, precision, require_gpu):
    """Residuals that form the face fluxes on the fly must give the same bits
    as the flux-array kernels (flux, coarsening, residual) in a full solve."""
    if case == "config1":
        probs = [configs.config1()]
    elif case == "config3":
        probs = [configs.config3()]
    else:
        probs = [configs.extend_hierarchy(configs.small_3d(seed=s), k=2) for s in (51, 52)]
    prm = dict(coarse_tol=1e-300, coarse_max_it=20, max_cycles=5)
    out = []
    for fused in (True, False):
        g = fac.FacContext(probs, params=prm, precision=precision)
        g.set_fused_residual(fused)
        conv, its, res = g.solve()
        out.append((its.copy(), res.copy(),
                    [g.download(U, i, ln) for i in range(len(probs)) for ln in range(probs[0].nlev)]))
        g.close()
    assert np.array_equal(out[0][0], out[1][0])
    assert np.array_equal(out[0][1], out[1][1])
    for a, b in zip(out[0][2], out[1][2]):
        assert np.array_equal(a, b)


@pytest.mark.gpu
def test_autotune_keeps_results(require_gpu):
    """The autotuner only changes how patches are cut into staged units:
    the solve after it gives the same bits as with the default units."""
    probs = [configs.extend_hierarchy(configs.small_3d(seed=s), k=2) for s in (61, 62)]
    prm = dict(coarse_tol=1e-300, coarse_max_it=20, max_cycles=6)
    out = []
    for tune in (True, False):
        g = fac.FacContext(probs, params=prm, precision="mixed")
        if tune:
            chosen, ms = g.autotune()
            assert chosen in (12288, 16384, 24576, 32768, 49152)
            assert g.stage_depth in (2, 3)
            assert ms.shape == (10,) and np.all(ms > 0)
        g.zero(U)
        conv, its, res = g.solve()
        out.append((its.copy(), res.copy(), [g.download(U, i, ln) for i in range(2)
                                             for ln in range(probs[0].nlev)]))
        g.close()
    assert np.array_equal(out[0][0], out[1][0]) and np.array_equal(out[0][1], out[1][1])
    for a, b in zip(out[0][2], out[1][2]):
        assert np.array_equal(a, b)


def _rel_l2(a_list, b_list):
    num = sum(float(np.sum((a - b) ** 2)) for a, b in zip(a_list, b_list))
    den = sum(float(np.sum(b ** 2)) for b in b_list)
    return (num / max(den, 1e-300)) ** 0.5


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("case", ["config1", "small_3d_mg", "config3"])
def test_fgmres_matches_fac_solution(case, precision, require_gpu):
    """FGMRES with the FAC cycle as preconditioner reaches the same 1e-10
    relative residual with no more preconditioner applications than FAC
    needs cycles, and the same solution to 1e-9 relative L2."""
    if case == "config1":
        probs = [configs.extend_hierarchy(configs.config1(), k=3)]
    elif case == "config3":
        probs = [configs.extend_hierarchy(configs.config3(), k=3)]
    else:
        probs = [configs.extend_hierarchy(configs.small_3d(seed=s), k=2) for s in (71, 72)]
    prm = dict(coarse_tol=1e-300, coarse_max_it=20, max_cycles=100)
    g = fac.FacContext(probs, params=prm, precision=precision)
    conv_f, its_f, res_f = g.solve()
    uf = [g.download(U, i, ln) for i in range(len(probs)) for ln in range(probs[0].nlev)]
    g.zero(U)
    conv_k, its_k, res_k = g.solve_fgmres(20)
    uk = [g.download(U, i, ln) for i in range(len(probs)) for ln in range(probs[0].nlev)]
    g.close()
    assert conv_f.all() and conv_k.all(), (its_f, res_f, its_k, res_k)
    assert (its_k <= its_f).all(), (its_k, its_f)
    assert _rel_l2(uk, uf) <= 1e-9


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("mk", [configs.config1, configs.config3])
def test_fgmres_matches_oracle_solution(mk, precision, require_gpu):
    """FGMRES(20) around the FAC cycle, on the hierarchy extended by fully
    covered coarser levels, converges to the oracle's solution of the
    original hierarchy: both solved to 1e-12 relative residual, the
    solutions agree to 1e-9 relative L2 over the original levels (the
    converged-solution bar of the mixed-precision method)."""
    p = mk()
    x = configs.extend_hierarchy(p, k=3)
    g = fac.FacContext([x], params=dict(coarse_tol=1e-300, coarse_max_it=20, max_cycles=100,
                                        relative_residual_tol=1e-12), precision=precision)
    conv, its, res = g.solve_fgmres(20)
    k = x.virtual_levels
    uk = [g.download(U, 0, ln + k) for ln in range(p.nlev)]
    g.close()
    assert conv[0], (its, res)
    op = Oracle(p, params=dict(coarse_tol=1e-12, relative_residual_tol=1e-12))
    assert op.solve()[0]
    assert _rel_l2(uk, [op.get(U, ln) for ln in range(p.nlev)]) <= 1e-9
