"""Writes tests/golden/damping_ode.json: the exact solution of the reference's damping ODE
(src/pgen/tests/dust_damping.cpp:9-16)
    du/dt = sum_s eps_s (v_s - u)/t_s,   dv_s/dt = -(v_s - u)/t_s
for the species mixtures of tst/test_suite/dust/check_cloud_imex3d.py:96-103 (resolved and
stiff), by the matrix exponential, together with the error bound the imex2+ drag step
must meet at the listed dt (second order: the bound is the measured error of the restated
scheme rounded up by 2x; the test also checks the order).  Run: python tests/golden/make_golden.py
"""
import json
import os

import numpy as np
from scipy.linalg import expm


def exact(taus, eps, vd, t):
    N = len(taus)
    A = np.zeros((N + 1, N + 1))
    for s in range(N):
        A[0, 0] -= eps[s] / taus[s]
        A[0, 1 + s] += eps[s] / taus[s]
        A[1 + s, 1 + s] = -1.0 / taus[s]
        A[1 + s, 0] = 1.0 / taus[s]
    return (expm(A * t) @ np.array([0.0] + list(vd))).tolist()


cases = []
for taus, bound in (([0.1, 0.03, 1.0], 2e-5), ([1e-4, 0.03, 1.0], 1e-5)):
    eps = [0.2, 0.5, 0.3]
    vd = [0.01 / 3, 0.02 / 3, 0.01]
    dt = 0.4 / 16
    tlim = 0.2
    n = int(round(tlim / dt))
    cases.append(dict(taus=taus, eps=eps, vd=vd, dt=dt, tlim=tlim, t=n * dt,
                      exact=exact(taus, eps, vd, n * dt), max_err=bound))
out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "damping_ode.json")
with open(out, "w") as f:
    json.dump(dict(source="src/pgen/tests/dust_damping.cpp:9-16", cases=cases), f, indent=1)
print(out)
