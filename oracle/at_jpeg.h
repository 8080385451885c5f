/* CPU checker of the JPEG input path. TEST INFRASTRUCTURE ONLY.

   oj_decode restates, for this project, the reference's baseline JPEG
   decoder (common/pjpeg.c of bouk/apriltags-fast, with the integer IDCT of
   common/pjpeg-idct.c:272-385) call for call in what it produces: the same
   marker walk, the same byte reader (FF00 unstuffing only, 1-bits past the
   end of the buffer), the same Huffman code space, the same restart check
   (which zeroes the DC predictor of the scan's first component only), the
   same component planes. It is pinned to the reference compiled from its
   own sources (oracle/_ref) by the CPU tests. Not linked into the product
   library. (The test inputs come from the package's synthetic-input
   encoder, apriltags_fast_b200/csrc/synth_jpeg.c.) */
#ifndef AT_JPEG_ORACLE_H
#define AT_JPEG_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* The reference's error codes (common/pjpeg.h:84-96). */
enum { OJ_OK = 0, OJ_ERR_FILE, OJ_ERR_DQT, OJ_ERR_SOF, OJ_ERR_DHT, OJ_ERR_SOS, OJ_ERR_MISSING_DHT,
       OJ_ERR_DRI, OJ_ERR_RESET, OJ_ERR_EOF, OJ_ERR_UNSUPPORTED };

/* The reference's flag: use the Annex K Huffman tables when the file
   carries none (common/pjpeg.h:79-82). */
enum { OJ_MJPEG = 2 };

typedef struct oj_plane {
    uint32_t width, height, stride;
    uint8_t *data;
    uint8_t id, hv, scalex, scaley, tq, tda;
} oj_plane;

typedef struct oj_image {
    uint32_t width, height;
    int ncomponents;
    oj_plane comp[3];
} oj_image;

/* Decodes buf into *out (component planes as the reference lays them
   out). Returns an OJ_* code; on error *out holds nothing to free. */
int oj_decode(const uint8_t *buf, int64_t len, uint32_t flags, oj_image *out);
void oj_free(oj_image *im);

/* Component 0 cropped to width x height, rows of `stride` bytes
   (pjpeg_to_u8_baseline). Returns 0, or -1 when the plane is smaller. */
int oj_gray(const oj_image *im, uint8_t *dst, int64_t stride);

#ifdef __cplusplus
}
#endif
#endif
