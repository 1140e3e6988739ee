"""Type ids, aggregation kinds and policies, numbered exactly as libcudf's
(cpp/include/cudf/types.hpp:201-233, cpp/include/cudf/aggregation.hpp:86-102)."""
from enum import IntEnum

import numpy as np
import torch


class TypeId(IntEnum):
    EMPTY = 0
    INT8 = 1
    INT16 = 2
    INT32 = 3
    INT64 = 4
    UINT8 = 5
    UINT16 = 6
    UINT32 = 7
    UINT64 = 8
    FLOAT32 = 9
    FLOAT64 = 10
    BOOL8 = 11
    TIMESTAMP_DAYS = 12
    TIMESTAMP_SECONDS = 13
    TIMESTAMP_MILLISECONDS = 14
    TIMESTAMP_MICROSECONDS = 15
    TIMESTAMP_NANOSECONDS = 16
    DURATION_DAYS = 17
    DURATION_SECONDS = 18
    DURATION_MILLISECONDS = 19
    DURATION_MICROSECONDS = 20
    DURATION_NANOSECONDS = 21


class Kind(IntEnum):
    SUM = 0
    PRODUCT = 1
    MIN = 2
    MAX = 3
    COUNT_VALID = 4
    COUNT_ALL = 5
    SUM_OF_SQUARES = 8
    MEAN = 9
    VARIANCE = 11
    STD = 12
    ARGMAX = 15
    ARGMIN = 16


class NullPolicy(IntEnum):
    EXCLUDE = 0
    INCLUDE = 1


class Sorted(IntEnum):
    NO = 0
    YES = 1


WIDTH = {TypeId.INT8: 1, TypeId.INT16: 2, TypeId.INT32: 4, TypeId.INT64: 8, TypeId.UINT8: 1,
         TypeId.UINT16: 2, TypeId.UINT32: 4, TypeId.UINT64: 8, TypeId.FLOAT32: 4,
         TypeId.FLOAT64: 8, TypeId.BOOL8: 1, TypeId.TIMESTAMP_DAYS: 4, TypeId.DURATION_DAYS: 4}
for _t in (13, 14, 15, 16, 18, 19, 20, 21):
    WIDTH[TypeId(_t)] = 8

TORCH_DTYPE = {
    TypeId.INT8: torch.int8, TypeId.INT16: torch.int16, TypeId.INT32: torch.int32,
    TypeId.INT64: torch.int64, TypeId.UINT8: torch.uint8, TypeId.UINT16: torch.uint16,
    TypeId.UINT32: torch.uint32, TypeId.UINT64: torch.uint64, TypeId.FLOAT32: torch.float32,
    TypeId.FLOAT64: torch.float64, TypeId.BOOL8: torch.bool,
    TypeId.TIMESTAMP_DAYS: torch.int32, TypeId.DURATION_DAYS: torch.int32,
}
for _t in (13, 14, 15, 16, 18, 19, 20, 21):
    TORCH_DTYPE[TypeId(_t)] = torch.int64

NUMPY_DTYPE = {
    TypeId.INT8: np.int8, TypeId.INT16: np.int16, TypeId.INT32: np.int32, TypeId.INT64: np.int64,
    TypeId.UINT8: np.uint8, TypeId.UINT16: np.uint16, TypeId.UINT32: np.uint32,
    TypeId.UINT64: np.uint64, TypeId.FLOAT32: np.float32, TypeId.FLOAT64: np.float64,
    TypeId.BOOL8: np.uint8, TypeId.TIMESTAMP_DAYS: np.int32, TypeId.DURATION_DAYS: np.int32,
}
for _t in (13, 14, 15, 16, 18, 19, 20, 21):
    NUMPY_DTYPE[TypeId(_t)] = np.int64

CAI_TYPESTR = {1: "|i1", 2: "<i2", 3: "<i4", 4: "<i8", 5: "|u1", 6: "<u2", 7: "<u4", 8: "<u8",
               9: "<f4", 10: "<f8", 11: "|b1"}
for _t in (12, 17):
    CAI_TYPESTR[_t] = "<i4"
for _t in (13, 14, 15, 16, 18, 19, 20, 21):
    CAI_TYPESTR[_t] = "<i8"

FROM_TORCH = {torch.int8: TypeId.INT8, torch.int16: TypeId.INT16, torch.int32: TypeId.INT32,
              torch.int64: TypeId.INT64, torch.uint8: TypeId.UINT8, torch.uint16: TypeId.UINT16,
              torch.uint32: TypeId.UINT32, torch.uint64: TypeId.UINT64,
              torch.float32: TypeId.FLOAT32, torch.float64: TypeId.FLOAT64, torch.bool: TypeId.BOOL8}
