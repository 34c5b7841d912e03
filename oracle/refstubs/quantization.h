/* stand-in for OpenGraph's quantization.h (absent from the reference
 * checkout): the helpers of the quantised pulls (pageRank.c:2119-2677),
 * restated from the published uniform affine scheme (Jacob et al., CVPR
 * 2018); not pinned.  min and max of the vector in one sequential sweep,
 * scale = (max - min) / (2^W - 1) in binary32, q = round-half-even(x / scale)
 * clamped to [0, 2^W - 1] plus the zero point (which the reference sets to
 * 0); a zero scale quantises everything to the zero point.  The unsuffixed
 * forms are only declared: their users (the push variants) are never linked
 * here. */
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

void getMinMax(struct quant_params *p, const float *x, uint32_t n);
float GetScale(float mn, float mx);
uint32_t quantize(float x, float scale, uint32_t zero);
#endif
