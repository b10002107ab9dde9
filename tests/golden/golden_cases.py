"""Cases whose oracle outputs are pinned in oracle_golden.json.

The reference has no golden vectors of its own, so these pin the oracle
against itself at commit time: any later change to the restatement that moves
a result beyond 1e-14 relative fails test_oracle.test_golden_vectors.
"""
from __future__ import annotations

import numpy as np


def compute_cases(oracle, pkg, table) -> dict:
    out = {}
    A, Z = pkg.configs.NET2
    oracle.network_init(A, Z)
    oracle.eos_init(table)
    states = [(1.0, 1e6), (1.0, 2.0e16), (1e4, 7.3e8), (3.0e-3, 4.1e4)]
    for n, (rho, T) in enumerate(states):
        st = oracle.eos(oracle.EOS_INPUT_RT, rho=rho, T=T, abar=6.4, zbar=3.2)
        out[f"eos_rt_{n}"] = [st.p, st.e, st.gam1, st.cs, st.dpdT, st.dedT, st.dpdr_e, st.dpde]
        re = oracle.eos(oracle.EOS_INPUT_RE, rho=rho, T=1e9, e=st.e * 1.5, abar=6.4, zbar=3.2)
        out[f"eos_re_{n}"] = [re.T, re.p, re.gam1, re.cs]
    for name, cfg in (("sedov16_outflow", pkg.configs.sedov64(scale=4, steps=2)),
                      ("ref8_periodic", pkg.configs.reference(scale=16, steps=2, max_box=4))):
        A, Z = cfg["network"]
        oracle.network_init(A, Z)
        oracle.eos_init(table)
        inst = cfg["instances"][0]
        lev, prob = oracle.level_from_instance(inst, pkg.configs.nvar(cfg))
        dts = [lev.coarse_step(-1.0) for _ in range(cfg["steps"])]
        G = oracle.assemble(lev, inst)
        out[name + "_dt"] = dts
        out[name + "_sums"] = [float(x) for x in G.reshape(-1, G.shape[3], order="F").sum(0)]
        out[name + "_probe"] = [float(x) for x in G[G.shape[0] // 2, 1, 2, :]]
    return out
