"""The CUDA library behind the checker interface used by golden_check.replay."""
import numpy as np

import aquarius_b200 as aq
from scenes import by_original

PARTICLE_FIELDS = ("position", "velocity_p", "fractions")


class LibChecker:
    """Stage 1 (grid-to-particle + advection) runs fused with the sort in the
    library; the reference's stage-1 output is in pre-sort order, so after
    stage 1 the particle fields are returned in pre-sort order."""

    def __init__(self, cfg):
        self.f = aq.Fluid(cfg)
        self.last = None

    def set_state(self, st):
        self.f.upload_state(st)

    def get_state(self, fields=None):
        want = None if fields is None else list(fields)
        if self.last == 1 and want is not None and "sort_index" not in want:
            want = want + ["sort_index"]
        st = self.f.download_state(want)
        if self.last == 1:
            for k in PARTICLE_FIELDS:
                if k in st:
                    st[k] = by_original(st[k], st["sort_index"])
        return st

    def stage(self, k):
        self.f.run_stage(k)
        self.last = k
