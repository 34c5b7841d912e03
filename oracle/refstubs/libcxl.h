/* stand-in for libcxl.h: the accelerator handle is opaque */
#ifndef REFSTUB_LIBCXL_H
#define REFSTUB_LIBCXL_H
struct cxl_afu_h;
#endif
