/* stand-in for OpenGraph's quantization.h (absent from the reference
 * checkout): the helpers of the quantised pulls and push
 * (pageRank.c:2119-2809), restated from the published uniform affine scheme
 * (Jacob et al., CVPR 2018); not pinned.  min and max of the vector in one
 * sequential sweep, scale = (max - min) / (2^W - 1) in binary32,
 * q = round-half-even(x / scale) clamped to [0, 2^W - 1] plus the zero point
 * (which the pulls set to 0); a zero scale quantises everything to the zero
 * point. */
#ifndef REFSTUB_QUANTIZATION_H
#define REFSTUB_QUANTIZATION_H
#include <math.h>
#include <stdint.h>
struct quant_params_32 { float scale; uint32_t zero; float min; float max; };
struct quant_params_16 { float scale; uint16_t zero; float min; float max; };
struct quant_params_8 { float scale; uint8_t zero; float min; float max; };
struct quant_params { float scale; uint32_t zero; float min; float max; };

#define REFSTUB_QUANT_FORMS(W)                                                              \
    static inline void getMinMax_##W(struct quant_params_##W *p, const float *x, uint32_t n) \
    {                                                                                       \
        float a = n ? x[0] : 0.0f, b = n ? x[0] : 0.0f;                                     \
        for (uint32_t i = 1; i < n; i++) {                                                  \
            if (x[i] < a)                                                                   \
                a = x[i];                                                                   \
            if (x[i] > b)                                                                   \
                b = x[i];                                                                   \
        }                                                                                   \
        p->min = a;                                                                         \
        p->max = b;                                                                         \
    }                                                                                       \
    static inline float GetScale_##W(float mn, float mx)                                    \
    {                                                                                       \
        return (mx - mn) / (float)((1ull << W) - 1);                                        \
    }                                                                                       \
    static inline uint##W##_t quantize_##W(float x, float scale, uint##W##_t zero)          \
    {                                                                                       \
        const uint64_t top = (1ull << W) - 1;                                               \
        float q;                                                                            \
        if (!(scale > 0.0f))                                                                \
            return zero;                                                                    \
        q = rintf(x / scale);                                                               \
        if (!(q > 0.0f))                                                                    \
            return zero;                                                                    \
        if (q >= (float)top)                                                                \
            return (uint##W##_t)(top + zero);                                               \
        return (uint##W##_t)((uint64_t)q + zero);                                           \
    }

REFSTUB_QUANT_FORMS(32)
REFSTUB_QUANT_FORMS(16)
REFSTUB_QUANT_FORMS(8)

/* the unsuffixed forms of the 32-bit push (pageRank.c:2725-2737): the same
 * as the 32-bit ones; GetZeroPoint's value is restated as 0, the zero point
 * the quantised pulls use */
static inline void getMinMax(struct quant_params *p, const float *x, uint32_t n)
{
    struct quant_params_32 q;
    getMinMax_32(&q, x, n);
    p->min = q.min;
    p->max = q.max;
}
static inline float GetScale(float mn, float mx) { return GetScale_32(mn, mx); }
static inline uint32_t GetZeroPoint(float mx, float scale)
{
    (void)mx;
    (void)scale;
    return 0;
}
static inline uint32_t quantize(float x, float scale, uint32_t zero) { return quantize_32(x, scale, zero); }
#endif
