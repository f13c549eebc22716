"""Shared seeded parity cases: geometry, CRS seed, DB, oracle precomp and
reference-client queries.  Conventions (all deterministic):

* CRS seed s: 64 bytes mt19937_64(s)() & 0xFF;
* DB: splitmix64(seed ^ k) mod 65535 at flat index k (row-major);
* queries: the reference client's query() with mt19937_64(rng_seed).
"""
import functools

import numpy as np

from oracle_lib import N, Oracle, RefLib, crs_seed_from, entry_slots


class Case:
    def __init__(self, n_entries, w, db_rows, crs=1, db_seed=0):
        self.o = Oracle()
        self.r = RefLib()
        self.geom = self.r.setup(n_entries, w, db_rows)
        _, _, self.R, self.C, self.G, self.D, self.ncts = self.geom
        self.n_entries, self.w, self.db_rows_arg = n_entries, w, db_rows
        self.seed = crs_seed_from(crs)
        self.db = self.o.fill_db(self.R * self.C, db_seed)
        self._pre = None

    @property
    def pre(self):
        if self._pre is None:
            self._pre = self.o.preprocess(self.seed, self.db, self.R, self.C, self.D)
        return self._pre

    def query(self, idx, rng_seed):
        return self.r.query(self.geom, self.seed, idx, rng_seed)

    def oracle_answer(self, qflat):
        dbe, pre = self.pre
        return self.o.answer(dbe, self.R, self.C, self.D, pre, qflat)

    def expected_slots(self, idx):
        return entry_slots(self.geom, self.db, idx)


@functools.lru_cache(maxsize=None)
def get_case(name):
    if name == "small":      # reference tests/test_e2e_gpu.cu:153-156 (n_packed = 1, no Horner)
        return Case(256, 120, 2048)
    if name == "medium":     # reference tests/test_e2e_gpu.cu:158-161 (n_packed = 4, Horner D = 4)
        return Case(262144, 120, 2048)
    if name == "batch":      # reference tests/test_gpu_batch.cu:26 (n_packed = 8)
        return Case(524288, 120, 2048, crs=7)
    if name == "cfg1":       # setup(65536, w=30): 32768 x 2048, CRS seed 1, DB seed 0
        return Case(65536, 30, 0, crs=1, db_seed=0)
    if name == "g128":       # 2048 x 262144 (1 GB DB), G = 128: the 16 GB geometry's group count
        return Case(8388608, 120, 2048, crs=3, db_seed=5)
    if name == "g512":       # 2048 x 1048576 (4.3 GB DB), G = 512 > D = 256: two response ciphertexts
        return Case(33554432, 120, 2048, crs=4, db_seed=6)
    raise KeyError(name)
