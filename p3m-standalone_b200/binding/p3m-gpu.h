/* p3mg-backed method tables for p3m-standalone's plugin interface
 * (method_t, types.h:306-316): drop p3m-gpu.c and this header into the
 * reference's source tree, add p3m-gpu.o to its OBJECTS and link libp3mg.so
 * (INTEGRATION.md gives the Makefile lines).  Each table keeps the id,
 * flags and error estimates of the CPU method it replaces. */
#ifndef P3M_GPU_H
#define P3M_GPU_H

#include "types.h"

extern const method_t method_p3m_ik_gpu;    /* replaces method_p3m_ik,   p3m-ik.c:46-49 */
extern const method_t method_p3m_ik_i_gpu;  /* replaces method_p3m_ik_i, p3m-ik-i.c:40-43 */
extern const method_t method_p3m_ad_gpu;    /* replaces method_p3m_ad,   p3m-ad.c:39-41 */
extern const method_t method_p3m_ad_i_gpu;  /* replaces method_p3m_ad_i, p3m-ad-i.c:39-41 */
extern const method_t method_p3m_ik_r_gpu;  /* replaces method_p3m_ik_r, p3m-ik-real.c:43-46 */
extern const method_t method_p3m_ad_r_gpu;  /* replaces method_p3m_ad_r, p3m-ad-real.c:39-41 */

/* FP64 (default) or FP32-mixed arithmetic for contexts created after the call. */
void p3m_gpu_set_precision(int precision);

/* Release the device context a GPU table's Init attached to d (the
 * counterpart of Free_data, p3m-common.c:234, for these tables). */
void p3m_gpu_free_data(data_t *d);

#endif
