"""Generates the golden fixtures in tests/golden/ from the reference itself.

Run where the reference tree exists (oracle/Makefile's REF, or $MKB_REFERENCE_TREE):
    python tests/golden/make_golden.py

* gauss_legendre.json -- the reference's generated Gauss-Legendre table
  (include/mikroptim/pupil/gauss_legendre_table.hpp), read as text: orders 1..16.
* singlet.npz   -- configuration-1 singlets (8 variants): residuals / OPD / status / merit
                   from residuals_cpu and merit_cpu, FD and adjoint Jacobians of 2 runs.
* objective.npz -- one configuration-2 objective at a reduced quadrature (3 rings x 6
                   spokes, soft failure): residuals, status, merit, adjoint and FD Jacobians.

The reference outputs come from oracle/_ref/libmko_ref.so, i.e. the reference's own CPU
sources compiled by oracle/Makefile. Inputs are regenerated from the seeded workload
generator, whose arrays are stored alongside so a change to the generator is detected.
"""

from __future__ import annotations

import json
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from mikroptim_b200 import workloads  # noqa: E402
from mikroptim_b200.batch import ResidualLayout  # noqa: E402
import oracle.pyoracle as po  # noqa: E402

TABLE = os.path.join(po.REFERENCE_TREE, "include/mikroptim/pupil/gauss_legendre_table.hpp")


def gauss_legendre_fixture() -> None:
    txt = open(TABLE).read()

    def numbers(name):
        body = re.search(name + r"\[136\] = \{(.*?)\};", txt, re.S).group(1)
        return [float(x) for x in re.findall(r"[-0-9.]+e[-+]?[0-9]+", body)]

    u, w = numbers("kGaussLegendreU"), numbers("kGaussLegendreW")
    out = {}
    for n in range(1, 17):
        off = n * (n - 1) // 2
        out[str(n)] = {"u": [repr(x) for x in u[off:off + n]],
                       "w": [repr(x) for x in w[off:off + n]]}
    with open(os.path.join(HERE, "gauss_legendre.json"), "w") as f:
        json.dump({"source": "include/mikroptim/pupil/gauss_legendre_table.hpp",
                   "orders": out}, f, indent=1)


def inputs_of(batch, x0):
    return dict(curvature=batch.curvature, thickness=batch.thickness, index=batch.index,
                pupil_radius=batch.pupil_radius, field_angle=batch.field_angle,
                field_target=batch.field_target, x0=x0)


def singlet_fixture(ref) -> None:
    b, st, vs, x0 = workloads.singlet(1024)
    b = b.subset(0, 8)
    x0 = x0[:8]
    lay = ResidualLayout(b.topology, st)
    res, opd, status = ref.residuals(b, lay)
    merit, failed, hard = ref.merit(b, lay)
    Jfd, r0fd, changes = ref.fd_jacobian(b.subset(0, 2), lay, vs, x0[:2])
    Jad, r0ad, stad = ref.adjoint_jacobian(b.subset(0, 2), lay, vs, x0[:2])
    np.savez_compressed(os.path.join(HERE, "singlet.npz"), **inputs_of(b, x0),
                        residuals=res, opd=opd, status=status, merit=merit, failed=failed,
                        hard_failed=hard, fd_jacobian=Jfd, fd_r0=r0fd, fd_changes=changes,
                        adjoint_jacobian=Jad, adjoint_r0=r0ad)


def objective_fixture(ref) -> None:
    b, st, vs, x0 = workloads.objective(4096, rings=3, spokes=6)
    b = b.subset(0, 2)
    x0 = x0[:2]
    lay = ResidualLayout(b.topology, st)
    res, opd, status = ref.residuals(b, lay)
    merit, failed, hard = ref.merit(b, lay)
    one = b.subset(0, 1)
    Jad, r0ad, stad = ref.adjoint_jacobian(one, lay, vs, x0[:1])
    Jfd, r0fd, changes = ref.fd_jacobian(one, lay, vs, x0[:1])
    np.savez_compressed(os.path.join(HERE, "objective.npz"), **inputs_of(b, x0),
                        residuals=res, opd=opd, status=status, merit=merit, failed=failed,
                        hard_failed=hard, adjoint_jacobian=Jad, adjoint_r0=r0ad,
                        fd_jacobian=Jfd, fd_r0=r0fd, fd_changes=changes)


if __name__ == "__main__":
    po.build()
    ref = po.reference()
    gauss_legendre_fixture()
    singlet_fixture(ref)
    objective_fixture(ref)
    for name in sorted(os.listdir(HERE)):
        print(name, os.path.getsize(os.path.join(HERE, name)))
