/* zarray_t: the growable array of the upstream AprilTag API, with the same
   layout and the same inline operations (common/zarray.h:42-50 of the
   reference), so code written against apriltag.h compiles unchanged. */
#pragma once
#include <assert.h>
#include <stddef.h>
#include <stdlib.h>
#include <string.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct zarray zarray_t;
struct zarray {
    size_t el_sz; /* bytes per element */
    int size;     /* elements in use */
    int alloc;    /* elements allocated */
    char *data;
};

static inline zarray_t *zarray_create(size_t el_sz) {
    assert(el_sz > 0);
    zarray_t *za = (zarray_t *)calloc(1, sizeof(zarray_t));
    za->el_sz = el_sz;
    return za;
}

static inline void zarray_destroy(zarray_t *za) {
    if (za == NULL) return;
    free(za->data);
    free(za);
}

static inline int zarray_size(const zarray_t *za) { return za->size; }

static inline void zarray_ensure_capacity(zarray_t *za, int capacity) {
    if (capacity <= za->alloc) return;
    int a = za->alloc < 8 ? 8 : za->alloc;
    while (a < capacity) a *= 2;
    za->data = (char *)realloc(za->data, (size_t)a * za->el_sz);
    za->alloc = a;
}

static inline void zarray_add(zarray_t *za, const void *p) {
    zarray_ensure_capacity(za, za->size + 1);
    memcpy(&za->data[(size_t)za->size * za->el_sz], p, za->el_sz);
    za->size++;
}

static inline void zarray_get(const zarray_t *za, int idx, void *p) {
    assert(idx >= 0 && idx < za->size);
    memcpy(p, &za->data[(size_t)idx * za->el_sz], za->el_sz);
}

static inline void zarray_get_volatile(const zarray_t *za, int idx, void *p) {
    assert(idx >= 0 && idx < za->size);
    *((void **)p) = &za->data[(size_t)idx * za->el_sz];
}

static inline void zarray_set(zarray_t *za, int idx, const void *p, void *outp) {
    assert(idx >= 0 && idx < za->size);
    if (outp != NULL) memcpy(outp, &za->data[(size_t)idx * za->el_sz], za->el_sz);
    memcpy(&za->data[(size_t)idx * za->el_sz], p, za->el_sz);
}

static inline void zarray_truncate(zarray_t *za, int sz) {
    assert(sz <= za->size);
    za->size = sz;
}

/* shuffle != 0: move the last element into the hole (order not kept) */
static inline void zarray_remove_index(zarray_t *za, int idx, int shuffle) {
    assert(idx >= 0 && idx < za->size);
    if (shuffle) {
        if (idx < za->size - 1)
            memcpy(&za->data[(size_t)idx * za->el_sz], &za->data[(size_t)(za->size - 1) * za->el_sz], za->el_sz);
    } else {
        memmove(&za->data[(size_t)idx * za->el_sz], &za->data[(size_t)(idx + 1) * za->el_sz],
                (size_t)(za->size - idx - 1) * za->el_sz);
    }
    za->size--;
}

static inline void zarray_clear(zarray_t *za) { za->size = 0; }

static inline zarray_t *zarray_copy(const zarray_t *za) {
    zarray_t *c = (zarray_t *)calloc(1, sizeof(zarray_t));
    c->el_sz = za->el_sz;
    zarray_ensure_capacity(c, za->size);
    if (za->size) memcpy(c->data, za->data, (size_t)za->size * za->el_sz);
    c->size = za->size;
    return c;
}

#ifdef __cplusplus
}
#endif
