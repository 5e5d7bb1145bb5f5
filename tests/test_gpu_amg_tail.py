"""The fused coarse-level launch of the AMG V-cycle at every size.

By default only levels of at most 4,096 rows run in the single
thread-block-cluster launch; PRISM_AMG_TAIL_ROWS moves that threshold (it is
read once per process, hence the subprocesses). With the whole hierarchy below
the finest level in the cluster launch, with none of it, and with the default,
the solutions must agree with the oracle within the solver tolerance of the
other AMG tests, in FP64 and in mixed precision."""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

from tests import cases

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SOL_TOL = 1e-8

SCRIPT = r"""
import json, sys
import numpy as np
sys.path.insert(0, {root!r})
import prism_b200
from prism_b200 import _abi as A, api
from tests import cases
out = {{}}
for prec in (A.PREC_FP64, A.PREC_MIXED):
    mesh, T, U, eqn = cases.transport_c3(24, prism_b200.lib(), conv="LinearUpwind")
    r = api.BiCGSTAB(precision=prec, krylov_tol=1e-12, preconditioner="amg").solve(eqn, 1, 0.0)
    np.save({path!r} + f"_{{prec}}.npy", T.values())
    out[prec] = [int(r.status), int(r.krylov_iterations)]
print(json.dumps(out))
"""


def _run(tmp_path, rows):
    path = str(tmp_path / f"tail{rows}")
    env = dict(os.environ)
    if rows is None:
        env.pop("PRISM_AMG_TAIL_ROWS", None)
    else:
        env["PRISM_AMG_TAIL_ROWS"] = str(rows)
    r = subprocess.run([sys.executable, "-c", SCRIPT.format(root=ROOT, path=path)], env=env, cwd=ROOT,
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    info = json.loads(r.stdout.strip().splitlines()[-1])
    return {int(k): (v, np.load(path + f"_{k}.npy")) for k, v in info.items()}


def test_tail_threshold_does_not_change_the_solution(tmp_path, orc):
    mesh, T, U, eqn = cases.transport_c3(24, orc, conv="LinearUpwind")
    from prism_b200 import api
    api.BiCGSTAB().solve(eqn, 1, 0.0)
    ref = T.values()
    for rows in (None, 0, 10 ** 9):
        for prec, ((status, its), sol) in _run(tmp_path, rows).items():
            err = cases.rel_l2(sol, ref)
            print(f"tail rows {rows} precision {prec}: {its} iterations, rel L2 vs oracle {err:.2e}")
            assert status == 0 and err < SOL_TOL
