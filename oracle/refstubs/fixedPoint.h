/* stand-in for OpenGraph's fixedPoint.h (absent from the reference checkout):
 * the two conversions of the 64-bit fixed-point pull
 * (pageRank.c:1276-1453).  The format is restated, not pinned: 32
 * fractional bits, conversion to fixed point truncating toward zero (the
 * accelerator's fixed-point contract also truncates and never rounds,
 * spmv_kernel_tb.sv:13-16), conversion back exact up to binary64 rounding.
 * The other fixed-point helpers of OpenGraph are not declared: their users
 * are never linked here. */
#ifndef REFSTUB_FIXEDPOINT_H
#define REFSTUB_FIXEDPOINT_H
#include <stdint.h>
#define SCALED64 32
#define DoubleToFixed64(x) ((uint64_t)(int64_t)((double)(x) * (double)(1ULL << SCALED64)))
#define Fixed64ToDouble(x) ((double)(int64_t)(x) / (double)(1ULL << SCALED64))
#endif
