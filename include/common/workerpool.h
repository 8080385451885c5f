/* The upstream detector keeps a workerpool_t pointer; the GPU detector has no
   CPU worker pool, so it stays NULL (apriltag.h:190 of the reference). */
#pragma once
typedef struct workerpool workerpool_t;
