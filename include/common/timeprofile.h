/* timeprofile_t of the upstream API (common/timeprofile.h:41-52 of the
   reference): apriltag_detector_detect stamps one entry per stage. */
#pragma once
#include <stdint.h>
#include <sys/time.h>
#include "zarray.h"

#ifdef __cplusplus
extern "C" {
#endif

struct timeprofile_entry {
    char name[32];
    int64_t utime;
};

typedef struct timeprofile timeprofile_t;
struct timeprofile {
    int64_t utime;
    zarray_t *stamps;
};

static inline int64_t utime_now(void) {
    struct timeval tv;
    gettimeofday(&tv, NULL);
    return (int64_t)tv.tv_sec * 1000000 + tv.tv_usec;
}

static inline timeprofile_t *timeprofile_create(void) {
    timeprofile_t *tp = (timeprofile_t *)calloc(1, sizeof(timeprofile_t));
    tp->stamps = zarray_create(sizeof(struct timeprofile_entry));
    tp->utime = utime_now();
    return tp;
}

static inline void timeprofile_destroy(timeprofile_t *tp) {
    if (tp == NULL) return;
    zarray_destroy(tp->stamps);
    free(tp);
}

static inline void timeprofile_clear(timeprofile_t *tp) {
    zarray_clear(tp->stamps);
    tp->utime = utime_now();
}

#ifdef __cplusplus
}
#endif
