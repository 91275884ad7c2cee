"""LP container in the reference's internal form.

Mirrors the fields of ``pramana::Model`` that the PDHG path reads
(src/core/model.h:24-64, src/core/sparse.h:11-16)::

    min  c^T x + offset
    s.t. row_lower <= A x <= row_upper
         col_lower <=   x <= col_upper

``A`` is stored column-major (CSC: ``start`` / ``index`` / ``value``) exactly
like ``pramana::SparseMatrix``.  Infinite bounds are +-inf (any |v| >= 1e20 is
treated as infinite, src/util/common.h:14).
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

INF_BOUND_THRESHOLD = 1e20


@dataclass
class Model:
    num_rows: int
    num_cols: int
    start: np.ndarray  # int32, num_cols + 1
    index: np.ndarray  # int32, nnz (row of each entry, increasing within a column)
    value: np.ndarray  # float64, nnz
    col_cost: np.ndarray
    col_lower: np.ndarray
    col_upper: np.ndarray
    row_lower: np.ndarray
    row_upper: np.ndarray
    obj_offset: float = 0.0
    name: str = "model"
    meta: dict = field(default_factory=dict)

    def __post_init__(self):
        self.start = np.ascontiguousarray(self.start, dtype=np.int32)
        self.index = np.ascontiguousarray(self.index, dtype=np.int32)
        self.value = np.ascontiguousarray(self.value, dtype=np.float64)
        for f in ("col_cost", "col_lower", "col_upper", "row_lower", "row_upper"):
            setattr(self, f, np.ascontiguousarray(getattr(self, f), dtype=np.float64))
        self.validate()

    @property
    def nnz(self) -> int:
        return int(self.start[-1]) if len(self.start) else 0

    def validate(self) -> None:
        m, n = self.num_rows, self.num_cols
        if len(self.start) != n + 1 or self.start[0] != 0:
            raise ValueError("start must have num_cols+1 entries and begin at 0")
        if np.any(np.diff(self.start) < 0):
            raise ValueError("start must be non-decreasing")
        nnz = self.nnz
        if len(self.index) != nnz or len(self.value) != nnz:
            raise ValueError("index/value must have start[-1] entries")
        if nnz and (self.index.min() < 0 or self.index.max() >= m):
            raise ValueError("row index out of range")
        for f, ln in (("col_cost", n), ("col_lower", n), ("col_upper", n), ("row_lower", m), ("row_upper", m)):
            if len(getattr(self, f)) != ln:
                raise ValueError(f"{f} must have length {ln}")
        if np.any(np.isnan(self.value)) or np.any(np.isnan(self.col_cost)):
            raise ValueError("NaN in model data")

    def row_activity(self, x: np.ndarray) -> np.ndarray:
        cols = np.repeat(np.arange(self.num_cols), np.diff(self.start))
        out = np.zeros(self.num_rows)
        np.add.at(out, self.index, self.value * x[cols])
        return out

    def objective(self, x: np.ndarray) -> float:
        return float(self.col_cost @ x) + self.obj_offset

    def csr(self):
        """(ptr, idx, val) of the row-major copy, each row in increasing column order."""
        order = np.lexsort((np.repeat(np.arange(self.num_cols), np.diff(self.start)), self.index))
        ptr = np.zeros(self.num_rows + 1, dtype=np.int32)
        np.cumsum(np.bincount(self.index, minlength=self.num_rows), out=ptr[1:])
        cols = np.repeat(np.arange(self.num_cols, dtype=np.int32), np.diff(self.start))
        return ptr, cols[order].astype(np.int32), self.value[order]


@dataclass
class LpCase:
    """One case of a family over a shared A (src/pdhg/pdhg.h:67-70).

    ``None`` means "same as the base model"."""
    cost: np.ndarray | None = None
    col_lower: np.ndarray | None = None
    col_upper: np.ndarray | None = None
    row_lower: np.ndarray | None = None
    row_upper: np.ndarray | None = None
