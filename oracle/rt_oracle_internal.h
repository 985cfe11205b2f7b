/* Test infrastructure only: declarations shared by rt_oracle.c and pt_oracle.c. */
#ifndef RT_ORACLE_INTERNAL_H
#define RT_ORACLE_INTERNAL_H
#include <stdint.h>

#include "rt_oracle.h"

/* Closest hit in the reference's traversal order, with the winner's offset and scaled
 * barycentrics b1 = e1/det, b2 = e2/det (Triangle.cu:562-566). */
void rto_trace_one_full(const rto_bvh *b, const float *o, const float *d, float tmax, int checkShadow,
                        int32_t *id, float *t, float *b1, float *b2);
void rto_triangle_vertices(const rto_bvh *b, uint32_t tri, float *v9);
uint32_t rto_bvh_ntri(const rto_bvh *b);

#endif
