"""Writes particle_restart_4.bin: a particle restart file in the layout of
NTLP's save_particles (particles.f90:1988-2046): int32 tnumpart, then one
352-byte record per droplet laid out as the MPI type particletype
(particles.f90:1930-1950): 4 int32 (pidx, procidx, nbr_pidx, nbr_procidx),
39 real8 in the declaration order of `type particle` (:76-85), int64 mult,
and two 8-byte pointers.  Built with numpy alone (independently of the
library under test).  Droplet 2 lies exactly on x = 0 and is dropped by
read_part_res's strict bounds test on a (0, 2) x (0, 2) domain.

Run: python tests/golden/make_restart_fixture.py
"""
from __future__ import annotations

import os

import numpy as np

REALS = (["vp1", "vp2", "vp3", "xp1", "xp2", "xp3", "uf1", "uf2", "uf3", "xrhs1", "xrhs2", "xrhs3",
          "vrhs1", "vrhs2", "vrhs3", "Tp", "Tprhs_s", "Tprhs_L", "Tf", "radius", "radrhs", "qinf", "qstar",
          "dist", "res", "m_s", "kappa_s", "rc", "actres", "numact", "u_sub1", "u_sub2", "u_sub3", "sigm_s",
          "vp_old1", "vp_old2", "vp_old3", "Tp_old", "radius_old"])
RECORD = np.dtype([("pidx", "<i4"), ("procidx", "<i4"), ("nbr_pidx", "<i4"), ("nbr_procidx", "<i4")]
                  + [(r, "<f8") for r in REALS] + [("mult", "<i8"), ("prev", "<u8"), ("next", "<u8")])
assert RECORD.itemsize == 352


def records(n: int = 4) -> np.ndarray:
    rec = np.zeros(n, dtype=RECORD)
    for i in range(n):
        rec["pidx"][i] = 101 + i
        rec["procidx"][i] = 3
        rec["nbr_pidx"][i] = 7
        rec["nbr_procidx"][i] = 1
        for k, name in enumerate(REALS):
            rec[name][i] = (k + 1) * 0.125 + i * 1.0e-3
        rec["xp1"][i] = 0.25 + 0.5 * i
        rec["xp2"][i] = 1.75 - 0.25 * i
        rec["xp3"][i] = 0.5 + 0.1 * i
        rec["radius"][i] = 1.0e-6 * (i + 1)
        rec["mult"][i] = 1000 + 17 * i
        rec["prev"][i] = 0x1111
        rec["next"][i] = 0x2222
    rec["xp1"][2] = 0.0          # on the domain edge: not read back
    return rec


def write(path: str, rec: np.ndarray) -> None:
    with open(path, "wb") as f:
        f.write(np.array([len(rec)], dtype="<i4").tobytes())
        f.write(rec.tobytes())


if __name__ == "__main__":
    write(os.path.join(os.path.dirname(os.path.abspath(__file__)), "particle_restart_4.bin"), records())
