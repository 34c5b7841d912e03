/* stand-in for OpenGraph's boolean.h */
#ifndef REFSTUB_BOOLEAN_H
#define REFSTUB_BOOLEAN_H
#ifndef TRUE
#define TRUE 1
#endif
#ifndef FALSE
#define FALSE 0
#endif
#endif
