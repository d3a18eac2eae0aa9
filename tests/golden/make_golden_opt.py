"""Makes tests/golden/opt_ref.npz from the REFERENCE's own GPU optimizer.

Runs on a GPU host with oracle/_ref/libfdref.so built (oracle/build_ref.sh):
    python tests/golden/make_golden_opt.py

The problem is tests/opt_cases.opt_case() (seeded; about 48k VOI rows x 1.9k
beamlets in 24 beams of 40-120 beamlets, 2.4M nonzeros).  Recorded, each from
the reference's code compiled unmodified or by line range:
- eval_g / eval_grad (IMRTOptUtils.cu:74-156, 512-631) at three fluences;
- proxL2Onehalf_QL_gpu (IMRTOptimize_var1.cu:457-570) with a zero-norm group
  and a group under the 1e-4 norm guard;
- beamWeightsInit_func, host and cuSPARSE forms (IMRTOptimize_var1.cu:49-161);
- one BOO_IMRT_L2OneHalf_gpu_QL run of 100 iterations (IMRTOptimize.cu:16-194)
  from the reference's initial fluence (srand(10086), :240-243);
- the beam-orientation loop BeamOrientationOptimization (:197-388): BOO phases
  ended by the prune triggers, each followed by DimReduction
  (IMRTOptUtils.cu:726-793), with the matrices of the kept beams coalesced as
  parallelMatCoalesce / diagBlock do (columns of the kept beams in order, D
  block diagonal) -- that glue is this script's, the arithmetic the reference's;
- FluencePolish (:479-601): polish_BOO_IMRT_gpu (:391-476) over the kept beams
  from the continued rand() stream.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [ROOT, os.path.dirname(HERE)]

import opt_cases  # noqa: E402
from oracle import ref  # noqa: E402
from fastdose_b200.optimize import reference_x0  # noqa: E402


def problem(case, A, D):
    w = case["w"]
    return ref.OptProblem(A, D, case["n_ptv"], case["n_oar"], w["max_dose"], w["max_weights"], w["min_dose"],
                          w["min_weights"], w["oar_weights"], case["gamma"], case["eta"])


def main(out=os.path.join(HERE, "opt_ref.npz")):
    case = opt_cases.opt_case()
    n, nb = case["n"], len(case["counts"])
    res = {}
    P = problem(case, case["A"], case["D"])
    pts = opt_cases.eval_points(case)
    res["eval_x"] = np.stack(pts)
    res["eval_g"] = np.array([P.eval_g(x) for x in pts], np.float32)
    gr = [P.eval_grad(x) for x in pts]
    res["eval_grad_value"] = np.array([v for v, _ in gr], np.float32)
    res["eval_grad"] = np.stack([g for _, g in gr])

    g0, tau = opt_cases.prox_input(case)
    res["prox_g0"], res["prox_tau"] = g0, tau
    res["prox"], res["prox_nrm"] = ref.opt_prox(case["masks"], g0, tau)

    res["weights_host"], res["weights_gpu"] = ref.opt_beam_weights(opt_cases.beam_blocks(case), case["n_ptv"],
                                                                   case["n_oar"])

    # the C library's rand() against the restatement the library ships
    x0 = ref.opt_rand01(n, 10086, reseed=True)
    assert np.array_equal(x0, reference_x0(n)), "this host's rand() differs from the restated glibc stream"

    b = opt_cases.BOO
    bw = (b["beam_weight"] * res["weights_host"]).astype(np.float32)
    r = P.boo(case["masks"], bw, x0, x0, b["step_size"], b["iters"], want=b["want"],
              change_trigger=b["change_trigger"])
    for k in ("loss", "x", "v", "nrm", "weights"):
        res["boo_" + k] = r[k]
    res["boo_scalars"] = np.array([r["k"], r["theta"], r["t"], r["active"], r["stop"]], np.float64)
    P.close()

    # BeamOrientationOptimization: phases, DimReduction, then FluencePolish
    o = opt_cases.OUTER
    active = list(range(nb))
    x = v = x0
    weights = (o["beam_weight"] * res["weights_host"]).astype(np.float32)
    state = (0, 0.0, o["step_size"])
    costs = np.zeros(o["max_iter"], np.float32)
    phases = []
    while True:
        A, D, masks = opt_cases.select(case, active)
        Q = problem(case, A, D)
        r = Q.boo(masks, weights, x, v, o["step_size"], o["max_iter"], prune=o["prune"], want=o["want"],
                  change_trigger=o["change_trigger"], state=state, loss=costs)
        Q.close()
        state = (r["k"], r["theta"], r["t"])
        phases.append((list(active), r["k"], r["active"]))
        act, weights, x, v = ref.opt_dim_reduction(active, case["counts"], r["weights"], r["x"], r["v"], r["nrm"],
                                                   int(r["active"]))
        active = [int(a) for a in act]
        if r["stop"]:
            break
    res["outer_costs"] = costs
    res["outer_active"] = np.array(active, np.int32)
    res["outer_x"], res["outer_v"], res["outer_weights"] = x, v, weights
    res["outer_scalars"] = np.array(state, np.float64)
    res["outer_phase_k"] = np.array([p[1] for p in phases], np.int32)
    res["outer_phase_active"] = np.array([p[2] for p in phases], np.float32)

    p = opt_cases.POLISH
    nk = int(sum(case["counts"][a] for a in active))
    xp = reference_x0(n + nk)[n:]  # arrayRand01 continues the stream seeded before the loop
    if not np.array_equal(xp, ref.opt_rand01(nk, reseed=False)):
        print("note: a library call drew from rand() during the loop; the polish start uses the restated stream")
    A, D, _ = opt_cases.select(case, active)
    Q = problem(case, A, D)
    r = Q.polish(xp, xp, p["step_size"], p["iters"])
    Q.close()
    res["polish_x0"], res["polish_loss"], res["polish_x"] = xp, r["loss"], r["x"]
    res["polish_scalars"] = np.array([r["k"], r["theta"], r["t"]], np.float64)

    np.savez_compressed(out, **res)
    print("wrote", out, {k: v.shape for k, v in res.items()})
    print("phases", phases, "kept", active)


if __name__ == "__main__":
    main(*sys.argv[1:])
