"""z-slab sharding on the GPU (timbir_b200/slab.py, mbir_set_z_slab): two
slabs of one volume run as two ranks (threads of this process on one GPU,
ThreadComm: they meet on the host between launches, no kernel waits on the
other rank) reach the whole volume's MAP estimate: the same cost (each
rank's cost is the whole volume's, summed through the all-reduce) and the
same image.  This checks the halo slices in the super-voxel and reference
ICD kernels and in the cost kernel, and the summed variance and convergence
ratio, against the unsharded stage of the same scan.

The exchange here is once per ICD iteration; the reference exchanges between
half-sweeps (XT_ICD_update.c:968-1058).  Both stop at the same fixed point,
so the comparison is at convergence: costs within 1e-6 relative (1e-5 with
the variance re-estimated), images within 1e-3 of the range (RMSE)."""
import threading

import numpy as np
import pytest

import timbir_b200
from timbir_b200 import slab, synth

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

PRIOR = dict(sig_s=0.002, sig_t=0.004, c_s=1.0, c_t=1.0, convg_thresh=0.0, remove_rings=0, quad_convex=1)


def scan_3d():
    return synth.ellipsoid_scan(48, 8, 72, I0=1e4, seed=21)


def scan_4d():
    s = synth.ellipsoid_scan(32, 8, 64, I0=1e4, seed=22)
    s.proj_angles = synth.interlaced_angles(4, 64, 32)
    s.proj_times = np.arange(64, dtype=np.float32)
    s.recon_times = np.array([0, 32, 64], np.float32)
    s.recon_num = 2
    return s


def make_stage(scan, schedule, prior, switches):
    st = timbir_b200.Stage(scan, **prior, blocks=2)
    if switches:
        st.set_switches(**switches)
    st.set_schedule(schedule)
    return st


def run_to_flat(step, cost, max_iters=600):
    """Iterate until two successive costs agree to 1e-11 relative."""
    prev = None
    for it in range(1, max_iters + 1):
        step(it)
        c = cost()
        if prev is not None and abs(prev - c) <= 1e-11 * abs(c):
            return c, it
        prev = c
    return c, max_iters


def whole(scan, schedule, prior, switches):
    st = make_stage(scan, schedule, prior, switches)
    st.prepare()
    c, n = run_to_flat(st.iterate, lambda: st.cost()[0])
    x = st.object()
    st.close()
    return c, x, n


def sharded(scan, schedule, prior, switches, ranks=2):
    stages = [make_stage(slab.split_scan(scan, r, ranks), schedule, prior, switches) for r in range(ranks)]
    comm = slab.ThreadComm(ranks, timeout=300)
    res, errs = [None] * ranks, []

    def run(r):
        try:
            s = slab.SlabSolver(stages[r], comm.for_rank(r))
            s.prepare()
            c, n = run_to_flat(s.iterate, lambda: s.cost()[0])
            res[r] = (c, stages[r].object(), n)
        except BaseException as e:  # reported below; the barrier releases the others
            errs.append(e)
            comm.barrier.abort()

    th = [threading.Thread(target=run, args=(r,)) for r in range(ranks)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    for st in stages:
        st.close()
    if errs:
        raise errs[0]
    return res


# case -> (scan, schedule, prior, switches, cost tolerance): the variance case
# (sigma^2 re-estimated each iteration jointly with the image) creeps to its
# fixed point more slowly, so both runs stop further from it; 1e-5 is the
# benchmark's MAP target
CASES = {
    "sv_3d": (scan_3d, 1, PRIOR, {}, 1e-6),
    "reference_3d": (scan_3d, 0, PRIOR, {}, 1e-6),
    "sv_4d_variance": (scan_4d, 1, dict(PRIOR, quad_convex=0), dict(update_var=1), 1e-5),
}


@pytest.mark.parametrize("case", sorted(CASES))
def test_two_slabs_reach_the_whole_volume_map(case):
    factory, schedule, prior, switches, tol = CASES[case]
    scan = factory()
    c_ref, x_ref, n_ref = whole(scan, schedule, prior, switches)
    res = sharded(scan, schedule, prior, switches)
    costs = [r[0] for r in res]
    assert costs[0] == costs[1]  # one whole-volume cost on every rank
    x = np.concatenate([r[1] for r in res], axis=1)
    rng = float(x_ref.max() - x_ref.min())
    rmse = float(np.sqrt(np.mean((x.astype(np.float64) - x_ref) ** 2)))
    print(f"{case}: whole {c_ref:.10g} ({n_ref} it), sharded {costs[0]:.10g} ({res[0][2]} it), "
          f"RMSE / range {rmse / rng:.2e}")
    assert abs(costs[0] - c_ref) <= tol * abs(c_ref)
    assert rmse < 1e-3 * rng


def test_sharded_stage_refuses_constraint_windows():
    scan = scan_3d()
    st = make_stage(slab.split_scan(scan, 0, 2), 1, dict(PRIOR, remove_rings=3), dict(update_proj_offset=3))
    st.set_z_slab(0, 2, lambda v: None)
    with pytest.raises(timbir_b200.MbirError):
        st.set_offset_windows(True)
    st.close()


def test_sharded_stage_is_refused_by_the_batch():
    scan = scan_3d()
    st = timbir_b200.Stage(slab.split_scan(scan, 1, 2), **PRIOR, blocks=2)
    st.set_batch_schedule(0, 1, 1)
    st.prepare()
    st.set_z_slab(1, 2, lambda v: None)
    with pytest.raises(timbir_b200.MbirError):
        timbir_b200.Batch([st])
    st.close()
