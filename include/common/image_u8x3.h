/* Interleaved RGB images of the upstream API (common/image_u8x3.h and
   common/image_types.h:46-55 of the reference): rows padded to a multiple
   of 192 bytes by default. */
#pragma once
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct image_u8x3 image_u8x3_t;
struct image_u8x3 {
    const int32_t width;
    const int32_t height;
    const int32_t stride; /* bytes per row */
    uint8_t *buf;
};

image_u8x3_t *image_u8x3_create(unsigned int width, unsigned int height);
image_u8x3_t *image_u8x3_create_alignment(unsigned int width, unsigned int height, unsigned int alignment);
void image_u8x3_destroy(image_u8x3_t *im);

#ifdef __cplusplus
}
#endif
