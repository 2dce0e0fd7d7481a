"""Generate tests/golden/presolve_golden.npz from pyRadMC's host pre-solve.

Run in a container where the reference package imports (``PYTHONPATH`` holding
its checkout):

    python tests/golden/make_presolve_golden.py /path/to/pyRadMC

It records, for the case of presolve_case.py:
  * the compiled stacks (BeamLimitingStack.flatten) and the mu tables the host
    pre-solve builds (geometry/head.py:119-180), so the device run needs no
    reference code;
  * chord lengths of random rays through each device (BeamLimitingStack.
    path_lengths, full line and forward half-line);
  * the totals of presolve_head (geometry/head.py:373-575) in the three
    configurations the reference's device test checks: attenuation, first
    Compton, first Compton with an air column.
"""

from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent.parent))


def main(ref_root: str) -> None:
    sys.path.insert(0, ref_root)
    from pyradmc.data.analytic import AnalyticCrossSections
    from pyradmc.geometry.collimation import MLC, BeamFrame, BeamLimitingStack, JawPair
    from pyradmc.geometry.head import AirColumn, _MuTables, presolve_head

    from tests.golden import presolve_case as case

    frame = BeamFrame(origin=case.FOCAL)
    stack = BeamLimitingStack(frame=frame, devices=(JawPair(**case.JAW), MLC(**case.MLC)))
    stack2 = BeamLimitingStack(frame=frame, devices=(JawPair(**case.JAW_U_FOCUSED), JawPair(**case.JAW_V),
                                                     MLC(**case.MLC_FOCUSED)))
    xs = AnalyticCrossSections()
    out: dict[str, np.ndarray] = {}
    for tag, st in (("s1", stack), ("s2", stack2)):
        c = st.flatten()
        for name in c.__dataclass_fields__:
            out[f"{tag}_{name}"] = np.asarray(getattr(c, name))
        out[f"{tag}_materials"] = np.asarray(st.materials)
        out[f"{tag}_densities"] = np.asarray(st.densities)
        p, d = case.random_rays(4000, seed=7 if tag == "s1" else 11)
        out[f"{tag}_ray_p"], out[f"{tag}_ray_d"] = p, d
        out[f"{tag}_len_full"] = st.path_lengths(p, d)
        out[f"{tag}_len_fwd"] = st.path_lengths(p, d, from_origin=True)
    source = case.FanSource()
    air = AirColumn(**case.AIR)
    pairs = (*zip(stack.materials, stack.densities, strict=True), (air.material, air.density))
    mu = _MuTables(xs, tuple(pairs), 0.010, source.max_energy, 512)
    out["mu_log_energy"] = mu._log_energies
    out["mu_log_total"] = mu._log_total
    out["mu_log_compton"] = mu._log_compton
    for tag, kw in (("att", dict(mode="attenuation", exit_z=case.EXIT_Z)),
                    ("fc", dict(mode="first_compton", exit_z=case.EXIT_Z)),
                    ("air", dict(mode="first_compton", exit_z=case.AIR_EXIT_Z, air=air))):
        ps = presolve_head(source, cross_sections=xs, n_histories=case.N, seed=case.SEED, stack=stack, **kw)
        c = ps.columns()
        w = c["weight"].astype(np.float64)
        e = c["energy"].astype(np.float64)
        kind = c["particle_type"]
        out[f"{tag}_totals"] = np.array([len(ps), w.sum(), (w * e).sum(), np.count_nonzero(kind == 1),
                                         np.count_nonzero(kind == 2), (w * e).sum() / w.sum(),
                                         (w * w).sum()])
        # weighted energy histograms per kind, for a spectral comparison
        bins = np.linspace(0.0, 6.0, 25)
        for k, name in ((1, "photon"), (2, "electron")):
            m = kind == k
            out[f"{tag}_{name}_hist"] = np.histogram(e[m], bins=bins, weights=w[m])[0]
            out[f"{tag}_{name}_hist2"] = np.histogram(e[m], bins=bins, weights=w[m] ** 2)[0]
    np.savez_compressed(HERE / "presolve_golden.npz", **out)
    print("wrote", HERE / "presolve_golden.npz", {k: v.shape for k, v in out.items() if k.endswith("totals")})


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
