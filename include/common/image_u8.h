/* Creating, reading and writing image_u8_t (common/image_u8.h:53-77 of the
   reference): rows are padded to a multiple of 96 bytes by default. */
#pragma once
#include "image_types.h"

#ifdef __cplusplus
extern "C" {
#endif

image_u8_t *image_u8_create_stride(unsigned int width, unsigned int height, unsigned int stride);
image_u8_t *image_u8_create(unsigned int width, unsigned int height);
image_u8_t *image_u8_create_alignment(unsigned int width, unsigned int height, unsigned int alignment);
image_u8_t *image_u8_create_from_pnm(const char *path);
image_u8_t *image_u8_copy(const image_u8_t *in);
void image_u8_destroy(image_u8_t *im);
int image_u8_write_pnm(const image_u8_t *im, const char *path);

#ifdef __cplusplus
}
#endif
