"""The PICellerator time step on one GPU handle, in the reference's order.

`_AbstractContext_Execute_Hook` (StGermain/Base/Context/src/AbstractContext.cxx:797-866)
hands each step the dt that the previous step's `_FiniteElementContext_PostSolve`
(StgFEM/SLE/SystemSetup/src/FiniteElementContext.cxx:345-395) computed after its solve
(0 before the first solve), adds it to currentTime after the step, and checkpoints after
that.  Inside the step the Stokes SLE is solved on the current points, the new dt is
computed from that velocity (`Stokes_SLE_UpdateDt`, the Courant limit), the material points
are advected by it with the same velocity (the SwarmAdvector time integrand, RK2 by
default: TimeIntegrator.cxx:190), and the integration swarm's update hook
(`_IntegrationPointsSwarm_UpdateHook`, PICellerator/MaterialPoints/src/
IntegrationPointsSwarm.cxx:391-460) re-maps the points and recalculates the weights — with
PCDVC that includes population control.  The initial remap (IntegrationPointsSwarm
initialise, :355-366) runs the same weights calculation once before the first step.

So a checkpoint written after step n holds the velocity and pressure of the n-th solve,
the points advected by that velocity (after population control), currentTime = the sum of
the dt handed to steps 1..n (the first is 0) and Dt = the dt computed after the n-th solve.
"""
from __future__ import annotations

from typing import Any, Dict, Optional

import numpy as np

from . import abi


def run_pic_steps(prob, uzawa: abi.UzawaParams, steps: int, pcdvc: Optional[Dict[str, Any]] = None,
                  weights_resolution=10, order: int = 2, precision: str = "fp64") -> Dict[str, Any]:
    """Run `steps` PIC time steps on a StokesProblem whose inputs are set (points, materials,
    BCs, body force).  `pcdvc` (PCDVC parameters with the reference's names) selects DVC
    weights with population control; None keeps constant weights.  Returns the last
    solution, the points, the time bookkeeping and per-step statistics."""
    if pcdvc is not None:
        prob.set_weights("dvc", weights_resolution)
    prob.locate()
    history = []
    if pcdvc is not None:
        history.append({"step": 0, "population_control": prob.population_control(**pcdvc)})
    t, dt = 0.0, 0.0
    u = p = None
    stats = {}
    for k in range(1, steps + 1):
        t_step = t
        prob.build_operator(precision)
        u, p, stats = prob.solve(uzawa)
        dt_next = prob.courant_dt(u)
        prob.advect(dt_next, u, order)
        prob.locate()
        rec = {"step": k, "time": t_step, "dt": dt, "uzawa": stats}
        if pcdvc is not None:
            rec["population_control"] = prob.population_control(**pcdvc)
        history.append(rec)
        t = t_step + dt      # currentTime += the dt handed to this step
        dt = dt_next
    coords, material, _ = prob.points()
    return {"u": u, "p": p, "coords": coords, "material": material, "current_time": t, "dt": dt,
            "history": history}
