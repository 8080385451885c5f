/* image_u8_t of the upstream API (common/image_types.h:36-44 of the
   reference). */
#pragma once
#include <stdint.h>

typedef struct image_u8 image_u8_t;
struct image_u8 {
    const int32_t width;
    const int32_t height;
    const int32_t stride;
    uint8_t *buf;
};
