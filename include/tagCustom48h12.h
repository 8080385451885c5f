/* The tagCustom48h12 family in the upstream API (tagCustom48h12.h of the reference): the codes are
   the library's built-in table; destroy frees only what create allocated. */
#pragma once
#include "apriltag.h"

#ifdef __cplusplus
extern "C" {
#endif

apriltag_family_t *tagCustom48h12_create(void);
void tagCustom48h12_destroy(apriltag_family_t *tf);

#ifdef __cplusplus
}
#endif
