"""Aggregation factories, named after pylibcudf.aggregation
(python/cudf/cudf/_lib/pylibcudf/aggregation.pyx:143-367) and
cudf::make_*_aggregation (cpp/include/cudf/aggregation.hpp:257-306)."""
from __future__ import annotations

from dataclasses import dataclass

from .types import Kind, NullPolicy


@dataclass(frozen=True)
class Aggregation:
    kind: Kind
    param: int = 0

    def __repr__(self):
        return f"Aggregation({self.kind.name}{', ddof=%d' % self.param if self.kind in (Kind.VARIANCE, Kind.STD) else ''})"


def sum() -> Aggregation:  # noqa: A001 - libcudf's name
    return Aggregation(Kind.SUM)


def product() -> Aggregation:
    return Aggregation(Kind.PRODUCT)


def min() -> Aggregation:  # noqa: A001
    return Aggregation(Kind.MIN)


def max() -> Aggregation:  # noqa: A001
    return Aggregation(Kind.MAX)


def count(null_handling: NullPolicy = NullPolicy.EXCLUDE) -> Aggregation:
    """COUNT_VALID for EXCLUDE, COUNT_ALL for INCLUDE (cudf::make_count_aggregation)."""
    return Aggregation(Kind.COUNT_ALL if null_handling == NullPolicy.INCLUDE else Kind.COUNT_VALID)


def mean() -> Aggregation:
    return Aggregation(Kind.MEAN)


def sum_of_squares() -> Aggregation:
    return Aggregation(Kind.SUM_OF_SQUARES)


def variance(ddof: int = 1) -> Aggregation:
    return Aggregation(Kind.VARIANCE, ddof)


def std(ddof: int = 1) -> Aggregation:
    return Aggregation(Kind.STD, ddof)


def argmax() -> Aggregation:
    return Aggregation(Kind.ARGMAX)


def argmin() -> Aggregation:
    return Aggregation(Kind.ARGMIN)
