/* Prints the sizes and field offsets of the upstream API structs; test_abi.py
   compiles it against include/ and compares with the reference's layout. */
#include <stdio.h>
#include <stddef.h>
#include "apriltag.h"
#include "apriltag_pose.h"
#include "common/pjpeg.h"
int main(void) {
    printf("family %zu ncodes %zu codes %zu wab %zu tw %zu rb %zu nbits %zu bx %zu by %zu h %zu name %zu impl %zu\n",
        sizeof(apriltag_family_t), offsetof(apriltag_family_t, ncodes), offsetof(apriltag_family_t, codes), offsetof(apriltag_family_t, width_at_border),
        offsetof(apriltag_family_t, total_width), offsetof(apriltag_family_t, reversed_border), offsetof(apriltag_family_t, nbits), offsetof(apriltag_family_t, bit_x),
        offsetof(apriltag_family_t, bit_y), offsetof(apriltag_family_t, h), offsetof(apriltag_family_t, name), offsetof(apriltag_family_t, impl));
    printf("detector %zu nthreads %zu qd %zu qs %zu re %zu ds %zu debug %zu qtp %zu tp %zu nedges %zu nsegments %zu nquads %zu tf %zu wp %zu mutex %zu fast %zu fb %zu fc %zu\n",
        sizeof(apriltag_detector_t), offsetof(apriltag_detector_t, nthreads), offsetof(apriltag_detector_t, quad_decimate), offsetof(apriltag_detector_t, quad_sigma),
        offsetof(apriltag_detector_t, refine_edges), offsetof(apriltag_detector_t, decode_sharpening), offsetof(apriltag_detector_t, debug), offsetof(apriltag_detector_t, qtp),
        offsetof(apriltag_detector_t, tp), offsetof(apriltag_detector_t, nedges), offsetof(apriltag_detector_t, nsegments), offsetof(apriltag_detector_t, nquads),
        offsetof(apriltag_detector_t, tag_families), offsetof(apriltag_detector_t, wp), offsetof(apriltag_detector_t, mutex), offsetof(apriltag_detector_t, fast),
        offsetof(apriltag_detector_t, family_bits), offsetof(apriltag_detector_t, families_changed));
    printf("detection %zu family %zu id %zu hamming %zu dm %zu H %zu c %zu p %zu\n", sizeof(apriltag_detection_t), offsetof(apriltag_detection_t, family),
        offsetof(apriltag_detection_t, id), offsetof(apriltag_detection_t, hamming), offsetof(apriltag_detection_t, decision_margin), offsetof(apriltag_detection_t, H),
        offsetof(apriltag_detection_t, c), offsetof(apriltag_detection_t, p));
    printf("qtp %zu zarray %zu matd %zu image_u8 %zu timeprofile %zu\n", sizeof(struct apriltag_quad_thresh_params), sizeof(zarray_t), sizeof(matd_t), sizeof(image_u8_t), sizeof(timeprofile_t));
    printf("info %zu det %zu tagsize %zu fx %zu fy %zu cx %zu cy %zu pose %zu R %zu t %zu\n", sizeof(apriltag_detection_info_t),
        offsetof(apriltag_detection_info_t, det), offsetof(apriltag_detection_info_t, tagsize), offsetof(apriltag_detection_info_t, fx),
        offsetof(apriltag_detection_info_t, fy), offsetof(apriltag_detection_info_t, cx), offsetof(apriltag_detection_info_t, cy),
        sizeof(apriltag_pose_t), offsetof(apriltag_pose_t, R), offsetof(apriltag_pose_t, t));
    printf("pjpeg %zu error %zu width %zu height %zu nc %zu comps %zu component %zu w %zu h %zu stride %zu data %zu id %zu hv %zu sx %zu sy %zu tq %zu tda %zu u8x3 %zu\n",
        sizeof(pjpeg_t), offsetof(pjpeg_t, error), offsetof(pjpeg_t, width), offsetof(pjpeg_t, height), offsetof(pjpeg_t, ncomponents),
        offsetof(pjpeg_t, components), sizeof(pjpeg_component_t), offsetof(pjpeg_component_t, width), offsetof(pjpeg_component_t, height),
        offsetof(pjpeg_component_t, stride), offsetof(pjpeg_component_t, data), offsetof(pjpeg_component_t, id), offsetof(pjpeg_component_t, hv),
        offsetof(pjpeg_component_t, scalex), offsetof(pjpeg_component_t, scaley), offsetof(pjpeg_component_t, tq), offsetof(pjpeg_component_t, tda),
        sizeof(image_u8x3_t));
    printf("errors %d %d %d %d flags %d %d\n", PJPEG_ERR_FILE, PJPEG_ERR_MISSING_DHT, PJPEG_ERR_RESET, PJEPG_ERR_UNSUPPORTED, PJPEG_STRICT, PJPEG_MJPEG);
    return 0;
}
