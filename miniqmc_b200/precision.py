"""Per-quantity error of one arithmetic form of the walker hot path against
another, on the same system, positions and random streams.

The mixed form (FP32 table, orbitals, distance rows, Jastrows, inverse and
Woodbury GEMMs; FP64 LU refresh, log-det and k x k block) is measured
against an FP64 form that evaluates the same FP32-rounded spline table in
FP64 (`QMC_FILL_UNIFORM_F32`), so the difference is the arithmetic alone.
The quantities follow what the reference's check drivers compare
(check_spo.cpp:246-340: SPO values, gradients, Hessians; check_wfc.cpp:
300-480: log value, gradients, ratios) plus the post-sweep log-det drift:
the log|det| accumulated through the accepted ratios
(DiracDeterminant::acceptMove, DiracDeterminant.cpp:129-146) against a fresh
FP64 evaluation at the same final positions.

Used by bench.py (its `error` field) and by tests/precision_report.py.
"""
import numpy as np


def stats(e):
    e = np.asarray(e, dtype=float).ravel()
    return {'median': float(np.median(e)), 'p99': float(np.percentile(e, 99)), 'max': float(e.max())}


def normwise(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def spo_errors(sys_test, sys_ref, points):
    """Norm-wise max error of V, G, H at Cartesian points [n][3]."""
    vt, gt, ht = sys_test.spo_vgh(points)
    vr, gr, hr = sys_ref.spo_vgh(points)
    return {'v_normwise': normwise(vt, vr), 'g_normwise': normwise(gt, gr), 'h_normwise': normwise(ht, hr)}


def _logdets(w):
    """log|det| of both spins accumulated by the batch, [W][2]."""
    return np.array(w.components()[:, :2])


def sweep_errors(w_test, w_ref, ur, de, checkpoints=(1,)):
    """Sweep both batches over the same host streams ur[S][W][1][N],
    de[S][W][1][N][3] (S MC steps, one substep each, acceptance 0.5, no
    refresh) and compare every move's ratio and gradient (the sweep trace)
    and, after each step listed in `checkpoints`, the log|det| each batch
    accumulated against a fresh FP64 evaluation of w_ref at the same
    positions.  The accept sequences must agree for the positions to be the
    same; `accept_sequence_identical` reports it.  `per_step` holds the
    log-ratio statistics of each step (the error grows from the fresh
    inverse of step 1 as the Woodbury updates accumulate)."""
    lt0, lr0 = w_test.evaluate_log(), w_ref.evaluate_log()
    out = {'logpsi_init_rel': float(np.max(np.abs(lt0 - lr0) / np.abs(lr0)))}
    n_steps = ur.shape[0]
    lr_err, g_err, same = [], [], True
    drift, per_step = {}, []
    for st in range(n_steps):
        rt = w_test.sweep(1, 1, 0.5, ur=ur[st:st + 1], delta=de[st:st + 1], trace=True)
        rr = w_ref.sweep(1, 1, 0.5, ur=ur[st:st + 1], delta=de[st:st + 1], trace=True)
        tt, tr = rt['trace'].reshape(-1, 8), rr['trace'].reshape(-1, 8)
        e = np.abs(np.log(np.abs(tt[:, 0])) - np.log(np.abs(tr[:, 0])))
        lr_err.append(e)
        per_step.append({'median': float(np.median(e)), 'p99': float(np.percentile(e, 99))})
        g_err.append(np.linalg.norm(tt[:, 1:4] - tr[:, 1:4], axis=1) /
                     np.maximum(np.linalg.norm(tr[:, 1:4], axis=1), 1e-300))
        same = same and bool(np.array_equal(tt[:, 7], tr[:, 7]))
        if st + 1 in checkpoints:
            acc_t, acc_r = _logdets(w_test), _logdets(w_ref)
            w_ref.evaluate_log()  # fresh FP64 log|det| at the (shared) positions
            fresh = _logdets(w_ref)
            drift[str(st + 1)] = {
                'test_rel_max': float(np.max(np.abs(acc_t - fresh) / np.abs(fresh))),
                'ref_rel_max': float(np.max(np.abs(acc_r - fresh) / np.abs(fresh))),
                'logpsi_rel_max': float(np.max(np.abs(rt['logpsi'] - rr['logpsi']) / np.abs(rr['logpsi'])))}
    out.update({'moves': int(sum(len(e) for e in lr_err)), 'log_ratio_abs': stats(np.concatenate(lr_err)),
                'log_ratio_abs_per_step': per_step,
                'grad_rel': stats(np.concatenate(g_err)), 'accept_sequence_identical': same,
                'logdet_drift_rel': drift})
    return out
