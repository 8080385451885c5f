/* The tagCircle21h7 family in the upstream API (tagCircle21h7.h of the reference): the codes are
   the library's built-in table; destroy frees only what create allocated. */
#pragma once
#include "apriltag.h"

#ifdef __cplusplus
extern "C" {
#endif

apriltag_family_t *tagCircle21h7_create(void);
void tagCircle21h7_destroy(apriltag_family_t *tf);

#ifdef __cplusplus
}
#endif
