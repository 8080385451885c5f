/* The tagStandard52h13 family in the upstream API (tagStandard52h13.h of the reference): the codes are
   the library's built-in table; destroy frees only what create allocated. */
#pragma once
#include "apriltag.h"

#ifdef __cplusplus
extern "C" {
#endif

apriltag_family_t *tagStandard52h13_create(void);
void tagStandard52h13_destroy(apriltag_family_t *tf);

#ifdef __cplusplus
}
#endif
