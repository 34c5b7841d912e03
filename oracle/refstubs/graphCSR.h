/* stand-in for OpenGraph's graphCSR.h: this repository's CSR container, the
 * one the library and its tests build */
#ifndef REFSTUB_GRAPHCSR_H
#define REFSTUB_GRAPHCSR_H
#include "../../include/graphCSR.h"
/* mask-mode id extraction; identity for ids without mask bits */
#ifndef EXTRACT_VALUE
#define EXTRACT_VALUE(x) (x)
#endif
#endif
