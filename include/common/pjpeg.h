/* Baseline JPEG decoding, the interface of the reference's common/pjpeg.h
   (common/pjpeg.h:28-103): same types, flags, error codes and calls. Here
   the entropy decoding and the IDCT run on the GPU (libapriltag_b200.so);
   the planes and images returned live in host memory, as the reference's
   do. at_jpeg_decode_gray (apriltag_fast.h) decodes straight into device
   frames for the detector. */
#pragma once
#include <stdint.h>

#include "image_u8.h"
#include "image_u8x3.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct pjpeg_component pjpeg_component_t;
struct pjpeg_component {
    /* resolution of this component's plane (whole MCUs) */
    uint32_t width, height;
    /* bytes per row (a multiple of 32) */
    uint32_t stride;
    /* data[y * stride + x] */
    uint8_t *data;

    uint8_t id;             /* component identifier */
    uint8_t hv;             /* horizontal (high 4 bits) and vertical sampling */
    uint8_t scalex, scaley; /* from hv */
    uint8_t tq;             /* quantisation table */
    uint8_t tda;            /* DC (high 4 bits) and AC Huffman tables of its last scan */
};

typedef struct pjpeg pjpeg_t;
struct pjpeg {
    int error;              /* non-zero: the decode failed */
    uint32_t width, height; /* pixels */
    int ncomponents;
    pjpeg_component_t *components;
};

enum PJPEG_FLAGS {
    PJPEG_STRICT = 1, /* accepted and ignored, as the reference does */
    PJPEG_MJPEG = 2,  /* files without Huffman tables use the ITU-T T.81 Annex K ones */
};

enum PJPEG_ERROR {
    PJPEG_OKAY = 0,
    PJPEG_ERR_FILE,        /* the file could not be read */
    PJPEG_ERR_DQT,         /* bad DQT segment */
    PJPEG_ERR_SOF,         /* bad SOF segment */
    PJPEG_ERR_DHT,         /* bad DHT segment */
    PJPEG_ERR_SOS,         /* bad SOS segment */
    PJPEG_ERR_MISSING_DHT, /* a scan needs a Huffman table never defined */
    PJPEG_ERR_DRI,         /* bad DRI segment */
    PJPEG_ERR_RESET,       /* a restart marker missing or out of sequence */
    PJPEG_ERR_EOF,         /* ran out of bytes */
    PJEPG_ERR_UNSUPPORTED, /* not a baseline sequential Huffman JPEG */
};

pjpeg_t *pjpeg_create_from_file(const char *path, uint32_t flags, int *error);
pjpeg_t *pjpeg_create_from_buffer(uint8_t *buf, int buflen, uint32_t flags, int *error);
void pjpeg_destroy(pjpeg_t *pj);

image_u8_t *pjpeg_to_u8_baseline(pjpeg_t *pj);
image_u8x3_t *pjpeg_to_u8x3_baseline(pjpeg_t *pj);

#ifdef __cplusplus
}
#endif
