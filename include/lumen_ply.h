/*
 * lumen_ply.h - Gaussian scenes from Stanford PLY files, straight to the
 * device SoA layout of LumenGpuGaussians.
 *
 * Reference readers (paths relative to the reference project):
 *   read_ply_ascii, src/scene/ply.mojo:73-138 (ASCII; columns x y z f_dc_0..2
 *     opacity scale_0..2 rot_0..3 taken by position; DC colour only)
 *   GaussianCloud.load_ply, python/lumen/cloud.py:163-199 (ASCII; columns
 *     x y z scale_0..2 rot_0..3 opacity f_dc_0..2 by position; DC only)
 * Both read the columns their own writers declare (ply.mojo:32-70,
 * cloud.py:131-161). Here columns are found by property name in the header,
 * which reads both of those files and the common 3D Gaussian splatting
 * training layout (binary, f_rest_* higher-order SH stored channel-major,
 * log-scales and opacity logits).
 *
 * SH: sh[i*48 + k*3 + ch] = f_dc_ch for k = 0 and f_rest[ch * m + k - 1]
 * for k >= 1 (m = f_rest count / 3); coefficients the file lacks are 0.
 * Quaternions: rot_0..3 = (w, x, y, z). Values are stored as in the file:
 * log_values tells whether scales are log-scales and opacities logits
 * (render with params_are_logits = log_values).
 */
#ifndef LUMEN_PLY_H
#define LUMEN_PLY_H

#include "lumen_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

#define LUMEN_PLY_VALUES_AUTO 0     /* log values when the file has f_rest_* properties, else linear */
#define LUMEN_PLY_VALUES_LINEAR 1
#define LUMEN_PLY_VALUES_LOG 2

typedef struct {
    int64_t count;                  /* vertices */
    int32_t binary;                 /* 1: binary_little_endian, 0: ascii */
    int32_t sh_degree;              /* 0..3, from the f_rest properties present */
    int32_t log_values;             /* 1: scale_* are log-scales and opacity is a logit */
    int32_t vertex_stride;          /* bytes per vertex (binary files) */
    int64_t data_offset;            /* bytes before the vertex data */
} LumenPlyInfo;

/* Read the header only. LUMEN_ERROR_IO_FAILURE when the file cannot be read,
 * LUMEN_ERROR_INVALID_ARGUMENT when it is not a Gaussian PLY this reader
 * supports (big-endian, a missing x/y/z/scale/rot/opacity/f_dc property, or
 * one of those not float32 in a binary file). */
LumenStatus lumen_ply_info(const char* path, int32_t values, LumenPlyInfo* info);

/* Load into host SoA arrays of at least info.count Gaussians (capacity). */
LumenStatus lumen_ply_load_host(const char* path, int32_t values, float* means, float* scales, float* quats,
                                float* opacities, float* sh, int64_t capacity, LumenPlyInfo* info);

/* Load into the device arrays of dst (dst->count = their capacity in
 * Gaussians; set to the number loaded). Binary vertex data is copied to the
 * device in chunks through page-locked memory and de-interleaved by a kernel;
 * ASCII files are parsed on the host. Waits. */
LumenStatus lumen_ply_load_device(const char* path, int32_t values, LumenGpuGaussians* dst, LumenPlyInfo* info,
                                  void* stream);

#ifdef __cplusplus
}
#endif

#endif /* LUMEN_PLY_H */
