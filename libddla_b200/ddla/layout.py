"""Process-grid layout -- mirror of the reference's python/ddla/layout.py.

The library serves the 1x1 grid: without mpi4py the communicator is the C
ABI's single-rank world, and any explicit grid other than 1x1 is rejected by
ddla_c_set with BACKEND_UNAVAILABLE.
"""
from __future__ import annotations

import math
from typing import Optional


class ProcessorLayout:
    def __init__(self, comm=None, np_rows: Optional[int] = None, np_cols: Optional[int] = None, major: str = "R"):
        self.major = major.upper()
        if self.major not in ("R", "C"):
            raise ValueError(f"Major must be 'R' (row-major) or 'C' (column-major), got {major}")
        from ._c_api import ddla_c_comm_rank, ddla_c_comm_size, ddla_c_default_comm

        self.comm = comm
        if comm is not None and hasattr(comm, "py2f"):
            self._comm_f = comm.py2f()
            self.nprocs = comm.Get_size()
            self.rank = comm.Get_rank()
        else:
            self._comm_f = int(comm) if isinstance(comm, int) else ddla_c_default_comm()
            self.rank = ddla_c_comm_rank(self._comm_f)
            self.nprocs = ddla_c_comm_size(self._comm_f)
        if np_rows is not None and np_cols is not None:
            self.np_rows, self.np_cols = int(np_rows), int(np_cols)
        elif np_rows is not None:
            self.np_rows = int(np_rows)
            self.np_cols = max(1, self.nprocs // self.np_rows)
        elif np_cols is not None:
            self.np_cols = int(np_cols)
            self.np_rows = max(1, self.nprocs // self.np_cols)
        else:
            best = 1
            for r in range(int(math.sqrt(self.nprocs)), 0, -1):
                if self.nprocs % r == 0:
                    best = r
                    break
            self.np_rows, self.np_cols = best, self.nprocs // best
        if self.major == "R":
            self.my_prow, self.my_pcol = self.rank // self.np_cols, self.rank % self.np_cols
        else:
            self.my_prow, self.my_pcol = self.rank % self.np_rows, self.rank // self.np_rows

    @property
    def comm_f(self) -> int:
        return self._comm_f
