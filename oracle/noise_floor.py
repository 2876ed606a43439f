"""ORACLE tooling: spread of the SIMP cantilever 40x20x10 under the oracle switches for details of the
reference that cannot be observed here (Vector256.Sum lane order, glibc pow vs correctly rounded powers)."""
import sys, json
sys.path.insert(0, __import__('os').path.dirname(__import__('os').path.dirname(__import__('os').path.abspath(__file__))))
import numpy as np
from oracle import oracle as O
from mycel_b200 import workloads as W
m, o = W.simp_cantilever_40x20x10()
res = {}
for lane, pw in ((0, 0), (0, 1), (1, 0), (2, 0)):
    O.set_modes(lane, pw, threads=8)
    r = O.topopt_run(m, o)
    res[(lane, pw)] = r
    print(lane, pw, r.n_iters, r.records[-1]["compliance"], sum(x["solver_iterations"] for x in r.records), flush=True)
base = res[(0, 0)]
out = {}
for k, r in res.items():
    if k == (0, 0): continue
    c = max(abs(a["compliance"] - b["compliance"]) / abs(b["compliance"]) for a, b in zip(r.records, base.records))
    d = float(np.abs(r.rho_phys_active - base.rho_phys_active).max())
    u = float(np.abs(r.u - base.u).max() / np.abs(base.u).max())
    its = [a["solver_iterations"] - b["solver_iterations"] for a, b in zip(r.records, base.records)]
    out[str(k)] = dict(max_rel_compliance=c, max_abs_rho_phys=d, max_rel_u=u, pcg_iter_diffs=its)
    print(k, out[str(k)], flush=True)
json.dump(out, open('noise_floor.json', 'w'), indent=1)
