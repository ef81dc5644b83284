"""Regenerates the committed golden fixtures of tests/golden/ from the
oracle (oracle/, the CPU restatement of the reference Fortran).

The reference repository ships no tests or golden vectors for this path and
no Fortran compiler exists on these machines, so these fixtures pin the
oracle itself: the GPU parity tests compare against them and against a live
oracle run.  Inputs are the seeded synthetic workloads of
radtrancode_b200/synth.py; a checksum of the input arrays is stored so that
a change of the generator is detected instead of silently comparing
different inputs.

    python tests/golden/make_golden.py
"""
import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import pyoracle as po  # noqa: E402
from radtrancode_b200 import synth  # noqa: E402


def input_digest(kt, cia, job) -> str:
    h = hashlib.sha256()
    for a in (kt.lnp, kt.tk, kt.delg, kt.data, cia.temps, cia.kcia, job.press, job.temp, job.delh, job.pp,
              job.amount, job.layinc, job.scale, job.emtemp, job.dte, job.dam, job.xmap, job.vwave):
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def cases():
    yield "c1", synth.config1()
    yield "c2s", synth.config2(nwave=8, nlayer=30, nbin=8)


def detexp_inputs():
    rng = np.random.default_rng(7)
    x = np.concatenate([np.linspace(-103.0, 88.0, 4001), rng.uniform(-12.0, 8.0, 4000),
                        np.array([0.0, -0.0, 1e-8, -1e-8, 88.7, -87.3])]).astype(np.float32)
    return x


def main():
    po.build()
    for name, (kt, cia, job) in cases():
        (c, g, gt), (perm, split, ties) = po.cirsrtfg_wave(kt, cia, job, po.ORC_MIXED, debug=True)
        c64, g64, gt64 = po.cirsrtfg_wave(kt, cia, job, po.ORC_FP64)
        extra = {}
        if perm is not None:
            extra = dict(split=split, ties=ties, perm_sha256=hashlib.sha256(perm.tobytes()).hexdigest())
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), input_sha256=input_digest(kt, cia, job),
                            calcout=c, gradients=g, gradtsurf=gt, calcout64=c64, gradients64=g64,
                            gradtsurf64=gt64, **extra)
        print(name, "written")
    x = detexp_inputs()
    np.savez_compressed(os.path.join(HERE, "detexp.npz"), x=x, y=po.det_expf(x))
    print("detexp written")


if __name__ == "__main__":
    main()
