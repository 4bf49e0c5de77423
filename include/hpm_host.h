/*
 * Host-side helpers of the command-line driver (libhpm_host.so): image
 * decoding for the dense folder's images/%08d.jpg, which the reference reads
 * with cv::imread(..., IMREAD_COLOR) (main.cpp:123-126, 212-213), and the
 * point-cloud files of its fusion.  No CUDA.
 */
#ifndef HPM_HOST_H
#define HPM_HOST_H

#include <stddef.h>
#include <stdint.h>

#include "hpm_types.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Decode PNG or baseline/extended-sequential JPEG bytes (format sniffed from
 * the content) to 8-bit BGR, w*h*3 bytes allocated with malloc into *bgr;
 * release with hpm_free_image.  Returns 0, or -1 with hpm_image_error() set. */
int hpm_decode_image(const uint8_t *bytes, size_t n, uint8_t **bgr, int *w, int *h);
void hpm_free_image(uint8_t *bgr);
const char *hpm_image_error(void);

/* Write fused points (hpm_fuse / hpm_get_points) to a PLY file as the
 * reference does.  fused == 0: ExportPointCloud (HPM.cpp:444-498), every point,
 * x y z and red green blue as (char)(int) of the BGR colour, non-finite
 * coordinates written as 0.  fused != 0: ExportFusedPointCloud (HPM.cpp:410-442),
 * points with finite coordinates and a non-zero normal, x y z, the normal made
 * unit in double, and the colour clamped to 0..255; *written (may be null)
 * receives their count.  Returns 0, or -1 when the file cannot be written. */
int hpm_write_ply(const char *path, const hpm_point *pts, size_t n, int fused, size_t *written);

#ifdef __cplusplus
}
#endif

#endif /* HPM_HOST_H */
