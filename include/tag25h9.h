/* The tag25h9 family in the upstream API (tag25h9.h of the reference): the codes are
   the library's built-in table; destroy frees only what create allocated. */
#pragma once
#include "apriltag.h"

#ifdef __cplusplus
extern "C" {
#endif

apriltag_family_t *tag25h9_create(void);
void tag25h9_destroy(apriltag_family_t *tf);

#ifdef __cplusplus
}
#endif
