/* matd_t: the upstream API's dense double matrix (common/matd.h:45-49 of the
   reference), as far as detections use it: the 3x3 homography H. */
#pragma once

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    unsigned int nrows, ncols;
    double *data; /* row-major */
} matd_t;

#define MATD_EL(m, row, col) (m)->data[((row) * (m)->ncols + (col))]

matd_t *matd_create(int rows, int cols);
matd_t *matd_create_data(int rows, int cols, const double *data);
matd_t *matd_copy(const matd_t *m);
void matd_destroy(matd_t *m);

#ifdef __cplusplus
}
#endif
