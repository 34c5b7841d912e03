/* stand-in for OpenGraph's fixedPoint.h (absent from the reference checkout):
 * the conversions of the fixed-point pulls (pageRank.c:1276-1991).  The
 * formats are restated, not pinned.
 * 64-bit: 32 fractional bits, conversion to fixed point truncating toward zero
 * (the accelerator's fixed-point contract also truncates and never rounds,
 * spmv_kernel_tb.sv:13-16), conversion back exact up to binary64 rounding.
 * 32/16/8-bit: W/2 fractional bits (Q16.16 is what the fixed-point SpMV
 * compute unit assumes of 32-bit operands, SCALEF = 16); to fixed point the
 * exact binary32 product truncated toward zero and kept modulo 2^W; back the
 * 64-bit sum rounded once to binary32 and scaled by 2^-(W/2).
 * The other fixed-point helpers of OpenGraph are not declared: their users
 * are never linked here. */
#ifndef REFSTUB_FIXEDPOINT_H
#define REFSTUB_FIXEDPOINT_H
#include <stdint.h>
#define SCALED64 32
#define DoubleToFixed64(x) ((uint64_t)(int64_t)((double)(x) * (double)(1ULL << SCALED64)))
#define Fixed64ToDouble(x) ((double)(int64_t)(x) / (double)(1ULL << SCALED64))
#define FloatToFixed32(x) ((uint32_t)(int64_t)((float)(x) * 65536.0f))
#define FloatToFixed16(x) ((uint16_t)(int64_t)((float)(x) * 256.0f))
#define FloatToFixed8(x) ((uint8_t)(int64_t)((float)(x) * 16.0f))
#define Fixed32ToFloat(x) ((float)(uint64_t)(x) / 65536.0f)
#define Fixed16ToFloat(x) ((float)(uint64_t)(x) / 256.0f)
#define Fixed8ToFloat(x) ((float)(uint64_t)(x) / 16.0f)
#endif
