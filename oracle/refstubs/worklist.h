/* stand-in for OpenGraph's worklist.h: byte-per-vertex worklists, as the
 * reference's data-driven variants use them (uint8_t arrays of
 * num_vertices entries, pageRank.c:2828-2838) */
#ifndef REFSTUB_WORKLIST_H
#define REFSTUB_WORKLIST_H
#include <stdint.h>
void resetWorkList(uint8_t *workList, uint32_t size);
void swapWorkLists(uint8_t **workList1, uint8_t **workList2);
#endif
