"""Python handle of the C ABI engine (mb_engine_*): resident star schema,
canonical index, rule planner and query execution.  A thin binding: every
query runs in libmerleb200.so."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import abi, check, lib


class Engine:
    def __init__(self, device: int = 0):
        self._e = C.c_void_p()
        check(lib().mb_engine_create(device, C.byref(self._e)))

    def close(self) -> None:
        if self._e:
            lib().mb_engine_destroy(self._e)
            self._e = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self) -> C.c_void_p:
        return self._e

    def gen_star(self, seed: int, k: int, nrows: int, width4: bool = False, row0: int = 0) -> None:
        check(lib().mb_engine_gen_star(self._e, seed, k, row0, nrows, 1 if width4 else 0))

    def load_star(self, h: abi.mb_star_host) -> None:
        check(lib().mb_engine_load_star(self._e, C.byref(h)))

    def build_index(self, probe_dims: bool = False) -> None:
        """Canonical index; probe_dims keeps the dimension probes through the
        foreign keys instead of the denormalised per-row columns."""
        check(lib().mb_engine_build_index_ex(self._e, abi.MB_INDEX_PROBE_DIMS if probe_dims else 0))

    def build_index_levels(self, level_mask: int, probe_dims: bool = False) -> None:
        """The index with only the levels of level_mask (mb_engine_plan_index)."""
        check(lib().mb_engine_build_index_levels(self._e, abi.MB_INDEX_PROBE_DIMS if probe_dims else 0,
                                                 level_mask))

    def plan_index(self, qs, budget_bytes: int) -> tuple[int, int, int]:
        """(level mask, index bytes, workload bytes) of the levels to keep
        within budget_bytes for the workload qs."""
        n = len(qs)
        qarr = (abi.mb_query * max(n, 1))(*qs)
        m, ib, wb = C.c_uint32(0), C.c_uint64(0), C.c_uint64(0)
        check(lib().mb_engine_plan_index(self._e, qarr, n, budget_bytes, C.byref(m), C.byref(ib), C.byref(wb)))
        return m.value, ib.value, wb.value

    def save_ssb(self, dirname) -> None:
        """The table as the reference's SSB column files (ssb_load's format)."""
        check(lib().mb_engine_save_ssb(self._e, str(dirname).encode()))

    def save_index(self, path) -> None:
        check(lib().mb_engine_save_index(self._e, str(path).encode()))

    def load_index(self, path, probe_dims: bool = False) -> None:
        """Index file written for this table (mb_engine_save_index)."""
        check(lib().mb_engine_load_index(self._e, str(path).encode(),
                                         abi.MB_INDEX_PROBE_DIMS if probe_dims else 0))

    def info(self) -> dict:
        i = abi.mb_engine_info()
        check(lib().mb_engine_get_info(self._e, C.byref(i)))
        return {f: getattr(i, f) for f, _ in i._fields_}

    @staticmethod
    def ngroups(q: abi.mb_query) -> int:
        return int(lib().mb_query_ngroups(C.byref(q)))

    def rule_plan(self, q: abi.mb_query) -> abi.mb_plan:
        p = abi.mb_plan()
        check(lib().mb_engine_plan_rule(self._e, C.byref(q), C.byref(p)))
        return p

    def query(self, q: abi.mb_query, plan: abi.mb_plan | None = None):
        """(int64 group sums, qualifying rows, stats) with results on the host."""
        ng = self.ngroups(q)
        out = np.zeros(max(ng, 1), np.int64)
        nq = C.c_uint64(0)
        st = abi.mb_query_stats()
        check(lib().mb_engine_query(self._e, C.byref(q), C.byref(plan) if plan is not None else None,
                                    out.ctypes.data, C.addressof(nq), C.byref(st)))
        return out[:ng], nq.value, st

    def query_batch(self, qs: list[abi.mb_query], opts: abi.mb_batch_opts | None = None):
        """Results of a batch through the batched scan (host buffers): the
        concatenated group sums (layout of mb_queries_layout) and row counts."""
        n = len(qs)
        qarr = (abi.mb_query * max(n, 1))(*qs)
        total = int(lib().mb_queries_layout(qarr, n, None))
        out = np.zeros(max(total, 1), np.int64)
        nq = np.zeros(max(n, 1), np.uint64)
        check(lib().mb_engine_query_batch(self._e, qarr, n, C.byref(opts) if opts is not None else None,
                                          out.ctypes.data, nq.ctypes.data))
        return out[:total], nq[:n]
