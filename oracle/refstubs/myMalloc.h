/* stand-in for OpenGraph's myMalloc.h */
#ifndef REFSTUB_MYMALLOC_H
#define REFSTUB_MYMALLOC_H
#include <stddef.h>
void *my_malloc(size_t size);
#endif
