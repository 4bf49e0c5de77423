/*
 * Host-side helpers of the command-line driver (libhpm_host.so): image
 * decoding for the dense folder's images/%08d.jpg, which the reference reads
 * with cv::imread(..., IMREAD_COLOR) (main.cpp:123-126, 212-213).  No CUDA.
 */
#ifndef HPM_HOST_H
#define HPM_HOST_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Decode PNG or baseline/extended-sequential JPEG bytes (format sniffed from
 * the content) to 8-bit BGR, w*h*3 bytes allocated with malloc into *bgr;
 * release with hpm_free_image.  Returns 0, or -1 with hpm_image_error() set. */
int hpm_decode_image(const uint8_t *bytes, size_t n, uint8_t **bgr, int *w, int *h);
void hpm_free_image(uint8_t *bgr);
const char *hpm_image_error(void);

#ifdef __cplusplus
}
#endif

#endif /* HPM_HOST_H */
