/* stand-in for OpenGraph's quantization.h (declared so that the quantized
 * variants compile; never called here) */
#ifndef REFSTUB_QUANTIZATION_H
#define REFSTUB_QUANTIZATION_H
#include <stdint.h>
struct quant_params_32 { float scale; uint32_t zero; float min; float max; };
struct quant_params_16 { float scale; uint16_t zero; float min; float max; };
struct quant_params_8 { float scale; uint8_t zero; float min; float max; };
struct quant_params { float scale; uint32_t zero; float min; float max; };
#endif
