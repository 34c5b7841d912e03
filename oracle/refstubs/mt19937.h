/* stand-in for OpenGraph's mt19937.h: the generator state carried in
 * struct Arguments (same shape as include/graphConfig.h of this repository) */
#ifndef REFSTUB_MT19937_H
#define REFSTUB_MT19937_H
#include <stdint.h>
#ifndef AG_MT19937_STATE_DEFINED
#define AG_MT19937_STATE_DEFINED
typedef struct mt19937state
{
    uint32_t mt[624];
    int32_t mti;
} mt19937state;
#endif
#endif
