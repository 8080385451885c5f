/* The tag36h10 family in the upstream API (tag36h10.h of the reference): the codes are
   the library's built-in table; destroy frees only what create allocated. */
#pragma once
#include "apriltag.h"

#ifdef __cplusplus
extern "C" {
#endif

apriltag_family_t *tag36h10_create(void);
void tag36h10_destroy(apriltag_family_t *tf);

#ifdef __cplusplus
}
#endif
