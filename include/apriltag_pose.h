/* Tag pose from a detection (apriltag_pose.h:1-79 of the reference): the
   same types and entry points, computed on the GPU (csrc/at_pose.cu). The
   results agree with the reference to rounding, not bit for bit: the 3x3
   algebra is grouped differently and the SVD is the library's own. */
#pragma once

#include "apriltag.h"
#include "common/matd.h"

#ifdef __cplusplus
extern "C" {
#endif

/* apriltag_pose.h:12-19 of the reference. */
typedef struct {
    apriltag_detection_t *det;
    double tagsize; /* metres */
    double fx;      /* pixels */
    double fy;
    double cx;
    double cy;
} apriltag_detection_info_t;

/* apriltag_pose.h:26-29 of the reference: the tag's pose in the camera frame. */
typedef struct {
    matd_t *R; /* 3x3 rotation */
    matd_t *t; /* 3x1 translation */
} apriltag_pose_t;

/* Replaces estimate_pose_for_tag_homography (apriltag_pose.c:455-488): the
   pose from the homography alone. */
void estimate_pose_for_tag_homography(apriltag_detection_info_t *info, apriltag_pose_t *pose);

/* Replaces estimate_tag_pose_orthogonal_iteration (apriltag_pose.c:490-526):
   the refined pose and its object-space error, and the second local minimum
   (pose2->R NULL and *err2 HUGE_VAL when there is none). */
void estimate_tag_pose_orthogonal_iteration(apriltag_detection_info_t *info, double *err1, apriltag_pose_t *pose1,
                                            double *err2, apriltag_pose_t *pose2, int nIters);

/* Replaces estimate_tag_pose (apriltag_pose.c:528-547): the better of the
   two; returns its object-space error. */
double estimate_tag_pose(apriltag_detection_info_t *info, apriltag_pose_t *pose);

#ifdef __cplusplus
}
#endif
