// Tag pose from a detection, on the device (apriltag_pose.c of the reference,
// with homography_to_pose of common/homography.c:275-350).
//
// Per detection (one thread each): the initial pose from the homography
// (its rotation made proper by a polar decomposition), refined by
// orthogonal iteration (Lu, Hager and Mjolsness 2000; apriltag_pose.c:43-141)
// over the tag's four corners; then the second local minimum of the
// object-space error (Schweighofer and Pinz 2006; apriltag_pose.c:259-452),
// refined the same way; the pose with the smaller error is the answer
// (apriltag_pose.c:528-547). Double precision throughout, as the
// reference; the operations are grouped differently (plain 3x3 algebra in
// registers instead of its matrix library, an own 3x3 SVD), so results
// agree with the reference to rounding (about 1e-12 relative), not bit for
// bit; the tests state their tolerance.
//
// Entry points: at_estimate_poses (all detections of the last detection
// call, one launch) and the reference's upstream estimate_tag_pose,
// estimate_tag_pose_orthogonal_iteration, estimate_pose_for_tag_homography
// (include/apriltag_pose.h), each one launch for one detection.
#include <cuda_runtime.h>
#include <math.h>
#include <stdio.h>
#include <string.h>

#include <vector>

#include "apriltag.h"
#include "apriltag_fast.h"
#include "apriltag_pose.h"

namespace {

struct V3 {
    double x, y, z;
};
struct M3 {
    double m[3][3];
};

__host__ __device__ inline V3 v3(double x, double y, double z) { return V3{x, y, z}; }
__host__ __device__ inline V3 add(V3 a, V3 b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
__host__ __device__ inline V3 sub(V3 a, V3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
__host__ __device__ inline V3 scale(V3 a, double s) { return v3(a.x * s, a.y * s, a.z * s); }
__host__ __device__ inline double dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__host__ __device__ inline V3 cross(V3 a, V3 b) {
    return v3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__host__ __device__ inline double comp(V3 a, int i) { return i == 0 ? a.x : i == 1 ? a.y : a.z; }
__host__ __device__ inline V3 mul(const M3 &A, V3 b) {
    return v3(A.m[0][0] * b.x + A.m[0][1] * b.y + A.m[0][2] * b.z, A.m[1][0] * b.x + A.m[1][1] * b.y + A.m[1][2] * b.z,
              A.m[2][0] * b.x + A.m[2][1] * b.y + A.m[2][2] * b.z);
}
__host__ __device__ inline M3 mul(const M3 &A, const M3 &B) {
    M3 C;
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) C.m[i][j] = A.m[i][0] * B.m[0][j] + A.m[i][1] * B.m[1][j] + A.m[i][2] * B.m[2][j];
    return C;
}
__host__ __device__ inline M3 transpose(const M3 &A) {
    M3 T;
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) T.m[i][j] = A.m[j][i];
    return T;
}
__host__ __device__ inline M3 identity() {
    M3 I = {};
    I.m[0][0] = I.m[1][1] = I.m[2][2] = 1.0;
    return I;
}
__host__ __device__ inline double det(const M3 &A) {
    return A.m[0][0] * (A.m[1][1] * A.m[2][2] - A.m[1][2] * A.m[2][1]) -
           A.m[0][1] * (A.m[1][0] * A.m[2][2] - A.m[1][2] * A.m[2][0]) +
           A.m[0][2] * (A.m[1][0] * A.m[2][1] - A.m[1][1] * A.m[2][0]);
}
__host__ __device__ inline M3 inverse(const M3 &A) {
    const double d = det(A);
    M3 B;
    B.m[0][0] = (A.m[1][1] * A.m[2][2] - A.m[1][2] * A.m[2][1]) / d;
    B.m[0][1] = (A.m[0][2] * A.m[2][1] - A.m[0][1] * A.m[2][2]) / d;
    B.m[0][2] = (A.m[0][1] * A.m[1][2] - A.m[0][2] * A.m[1][1]) / d;
    B.m[1][0] = (A.m[1][2] * A.m[2][0] - A.m[1][0] * A.m[2][2]) / d;
    B.m[1][1] = (A.m[0][0] * A.m[2][2] - A.m[0][2] * A.m[2][0]) / d;
    B.m[1][2] = (A.m[0][2] * A.m[1][0] - A.m[0][0] * A.m[1][2]) / d;
    B.m[2][0] = (A.m[1][0] * A.m[2][1] - A.m[1][1] * A.m[2][0]) / d;
    B.m[2][1] = (A.m[0][1] * A.m[2][0] - A.m[0][0] * A.m[2][1]) / d;
    B.m[2][2] = (A.m[0][0] * A.m[1][1] - A.m[0][1] * A.m[1][0]) / d;
    return B;
}
// v v' / (v' v): the projection onto the line of sight through v.
__host__ __device__ inline M3 line_projector(V3 v) {
    const double n = dot(v, v);
    const double c[3] = {v.x, v.y, v.z};
    M3 F;
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) F.m[i][j] = c[i] * c[j] / n;
    return F;
}

// The rotation closest to A (its polar factor U V'), from A's SVD: the
// eigenvectors V of A'A by cyclic Jacobi rotations, U = A V / sigma. A
// column of U whose singular value vanishes (A of rank 2, as the
// orthogonal iteration's cross-covariance of a planar tag always is) is
// the cross product of the other two.
__host__ __device__ inline M3 polar_rotation(const M3 &A) {
    M3 B = mul(transpose(A), A), V = identity();
    for (int sweep = 0; sweep < 40; sweep++) {
        const double off = B.m[0][1] * B.m[0][1] + B.m[0][2] * B.m[0][2] + B.m[1][2] * B.m[1][2];
        const double diag = B.m[0][0] * B.m[0][0] + B.m[1][1] * B.m[1][1] + B.m[2][2] * B.m[2][2];
        if (!(off > 1e-34 * diag)) break;
        for (int p = 0; p < 2; p++)
            for (int q = p + 1; q < 3; q++) {
                if (B.m[p][q] == 0.0) continue;
                const double theta = (B.m[q][q] - B.m[p][p]) / (2.0 * B.m[p][q]);
                const double t = (theta >= 0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
                const double c = 1.0 / sqrt(t * t + 1.0), s = t * c;
                for (int k = 0; k < 3; k++) {  // B <- J' B J
                    const double bkp = B.m[k][p], bkq = B.m[k][q];
                    B.m[k][p] = c * bkp - s * bkq;
                    B.m[k][q] = s * bkp + c * bkq;
                }
                for (int k = 0; k < 3; k++) {
                    const double bpk = B.m[p][k], bqk = B.m[q][k];
                    B.m[p][k] = c * bpk - s * bqk;
                    B.m[q][k] = s * bpk + c * bqk;
                }
                for (int k = 0; k < 3; k++) {  // V <- V J
                    const double vkp = V.m[k][p], vkq = V.m[k][q];
                    V.m[k][p] = c * vkp - s * vkq;
                    V.m[k][q] = s * vkp + c * vkq;
                }
            }
    }
    // singular values, largest first
    int ord[3] = {0, 1, 2};
    for (int i = 0; i < 3; i++)
        for (int j = i + 1; j < 3; j++)
            if (B.m[ord[j]][ord[j]] > B.m[ord[i]][ord[i]]) {
                const int t = ord[i];
                ord[i] = ord[j];
                ord[j] = t;
            }
    V3 vc[3], uc[3];
    double sig[3];
    for (int i = 0; i < 3; i++) {
        vc[i] = v3(V.m[0][ord[i]], V.m[1][ord[i]], V.m[2][ord[i]]);
        const double l = B.m[ord[i]][ord[i]];
        sig[i] = l > 0 ? sqrt(l) : 0.0;
    }
    uc[0] = scale(mul(A, vc[0]), 1.0 / sig[0]);
    uc[1] = scale(mul(A, vc[1]), 1.0 / sig[1]);
    if (sig[2] > 1e-9 * sig[0]) {
        uc[2] = scale(mul(A, vc[2]), 1.0 / sig[2]);
    } else {
        uc[2] = cross(uc[0], uc[1]);
    }
    // R = sum over k of u_k v_k'
    M3 R;
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
            double r = 0;
            for (int k = 0; k < 3; k++) r += comp(uc[k], i) * comp(vc[k], j);
            R.m[i][j] = r;
        }
    return R;
}

// The pose of the homography (common/homography.c:275-350 with fx negated,
// then the reference's axis flip and the tag's half size; apriltag_pose.c:
// 455-488): its rotation and translation. The column lengths are taken in
// single precision as the reference takes them (sqrtf).
__host__ __device__ inline void homography_pose(const double *H, double s2, double fx, double fy, double cx, double cy,
                                                M3 *R, V3 *t) {
    fx = -fx;
    double R20 = H[6], R21 = H[7], TZ = H[8];
    double R00 = (H[0] - cx * R20) / fx, R01 = (H[1] - cx * R21) / fx, TX = (H[2] - cx * TZ) / fx;
    double R10 = (H[3] - cy * R20) / fy, R11 = (H[4] - cy * R21) / fy, TY = (H[5] - cy * TZ) / fy;
    const double length1 = (double)sqrtf((float)(R00 * R00 + R10 * R10 + R20 * R20));
    const double length2 = (double)sqrtf((float)(R01 * R01 + R11 * R11 + R21 * R21));
    double s = 1.0 / (double)sqrtf((float)(length1 * length2));
    if (TZ > 0) s *= -1;
    R20 *= s, R21 *= s, TZ *= s, R00 *= s, R01 *= s, TX *= s, R10 *= s, R11 *= s, TY *= s;
    M3 A;
    A.m[0][0] = R00, A.m[0][1] = R01, A.m[0][2] = R10 * R21 - R20 * R11;
    A.m[1][0] = R10, A.m[1][1] = R11, A.m[1][2] = R20 * R01 - R00 * R21;
    A.m[2][0] = R20, A.m[2][1] = R21, A.m[2][2] = R00 * R11 - R10 * R01;
    const M3 P = polar_rotation(A);
    // the flip diag(1, -1, -1) on the left, and the tag's half size on t
    for (int j = 0; j < 3; j++) {
        R->m[0][j] = P.m[0][j];
        R->m[1][j] = -P.m[1][j];
        R->m[2][j] = -P.m[2][j];
    }
    *t = v3(TX * s2, -TY * s2, -TZ * s2);
}

// Orthogonal iteration over the 4 corners (apriltag_pose.c:43-141): R is
// the start and the result, t the result; returns the object-space error.
__host__ __device__ inline double orthogonal_iteration(const V3 *v, const V3 *p, V3 *t, M3 *R, int steps) {
    V3 pm = v3(0, 0, 0);
    for (int i = 0; i < 4; i++) pm = add(pm, p[i]);
    pm = scale(pm, 0.25);
    V3 pr[4];
    M3 F[4], avgF = {};
    for (int i = 0; i < 4; i++) {
        pr[i] = sub(p[i], pm);
        F[i] = line_projector(v[i]);
        for (int a = 0; a < 3; a++)
            for (int b = 0; b < 3; b++) avgF.m[a][b] += F[i].m[a][b];
    }
    M3 M1 = identity();
    for (int a = 0; a < 3; a++)
        for (int b = 0; b < 3; b++) M1.m[a][b] -= 0.25 * avgF.m[a][b];
    const M3 M1inv = inverse(M1);
    double error = HUGE_VAL;
    for (int it = 0; it < steps; it++) {
        V3 M2 = v3(0, 0, 0);
        for (int j = 0; j < 4; j++) {
            const V3 rp = mul(*R, p[j]);
            M2 = add(M2, sub(mul(F[j], rp), rp));
        }
        *t = mul(M1inv, scale(M2, 0.25));
        V3 q[4], qm = v3(0, 0, 0);
        for (int j = 0; j < 4; j++) {
            q[j] = mul(F[j], add(mul(*R, p[j]), *t));
            qm = add(qm, q[j]);
        }
        qm = scale(qm, 0.25);
        M3 M3c = {};
        for (int j = 0; j < 4; j++) {
            const V3 d = sub(q[j], qm);
            const double dc[3] = {d.x, d.y, d.z}, pc[3] = {pr[j].x, pr[j].y, pr[j].z};
            for (int a = 0; a < 3; a++)
                for (int b = 0; b < 3; b++) M3c.m[a][b] += dc[a] * pc[b];
        }
        *R = polar_rotation(M3c);
        if (det(*R) < 0)
            for (int a = 0; a < 3; a++) R->m[a][2] = -R->m[a][2];
        error = 0;
        for (int j = 0; j < 4; j++) {
            const V3 x = add(mul(*R, p[j]), *t);
            const V3 e = sub(x, mul(F[j], x));
            error += dot(e, e);
        }
    }
    return error;
}

__host__ __device__ inline double polyval(const double *c, int degree, double x) {
    double r = 0;
    for (int i = 0; i <= degree; i++) r += c[i] * pow(x, (double)i);
    return r;
}

// Real roots of a polynomial of degree D within +-1000 (apriltag_pose.c:
// 152-257): the roots of its derivative split the line into monotone
// pieces; each piece with a sign change is searched by Newton steps that
// fall back to bisection.
template <int D> struct PolyRoots {
    __host__ __device__ static int solve(const double *c, double *roots) {
        const double kMax = 1000;
        double d[D], droots[D];
        for (int i = 0; i < D; i++) d[i] = (i + 1) * c[i + 1];
        const int nd = PolyRoots<D - 1>::solve(d, droots);
        int n = 0;
        for (int i = 0; i <= nd; i++) {
            const double lo_x = i == 0 ? -kMax : droots[i - 1];
            const double hi_x = i == nd ? kMax : droots[i];
            const double flo = polyval(c, D, lo_x), fhi = polyval(c, D, hi_x);
            if (flo * fhi < 0) {
                double lower = flo < fhi ? lo_x : hi_x, upper = flo < fhi ? hi_x : lo_x;
                double root = 0.5 * (lower + upper), dx_old = upper - lower, dx = dx_old;
                double f = polyval(c, D, root), df = polyval(d, D - 1, root);
                for (int j = 0; j < 100; j++) {
                    if ((f + df * (upper - root)) * (f + df * (lower - root)) > 0 || fabs(2 * f) > fabs(dx_old * df)) {
                        dx_old = dx;
                        dx = 0.5 * (upper - lower);
                        root = lower + dx;
                    } else {
                        dx_old = dx;
                        dx = -f / df;
                        root += dx;
                    }
                    if (root == upper || root == lower) break;
                    f = polyval(c, D, root);
                    df = polyval(d, D - 1, root);
                    if (f > 0)
                        upper = root;
                    else
                        lower = root;
                }
                roots[n++] = root;
            } else if (fhi == 0) {
                roots[n++] = hi_x;
            }
        }
        return n;
    }
};
template <> struct PolyRoots<1> {
    __host__ __device__ static int solve(const double *c, double *roots) {
        if (fabs(c[0]) > 1000 * fabs(c[1])) return 0;
        roots[0] = -c[0] / c[1];
        return 1;
    }
};

__host__ __device__ inline M3 rows3(V3 a, V3 b, V3 c) {
    M3 M;
    M.m[0][0] = a.x, M.m[0][1] = a.y, M.m[0][2] = a.z;
    M.m[1][0] = b.x, M.m[1][1] = b.y, M.m[1][2] = b.z;
    M.m[2][0] = c.x, M.m[2][1] = c.y, M.m[2][2] = c.z;
    return M;
}

// The other local minimum of the object-space error, if there is one
// (apriltag_pose.c:259-452): false when none.
__host__ __device__ inline bool second_minimum(const V3 *v, const V3 *p, V3 t, const M3 &R, M3 *out) {
    const M3 I3 = identity();
    const V3 r3 = scale(t, 1.0 / sqrt(dot(t, t)));
    V3 r1 = sub(v3(1, 0, 0), scale(r3, r3.x));
    r1 = scale(r1, 1.0 / sqrt(dot(r1, r1)));
    const V3 r2 = cross(r3, r1);
    const M3 Rt = rows3(r1, r2, r3);
    const M3 R1p = mul(Rt, R);
    double r31 = R1p.m[2][0], r32 = R1p.m[2][1], hyp = sqrt(r31 * r31 + r32 * r32);
    if (hyp < 1e-100) r31 = 1, r32 = 0, hyp = 1;
    const M3 Rz = rows3(v3(r31 / hyp, -r32 / hyp, 0), v3(r32 / hyp, r31 / hyp, 0), v3(0, 0, 1));
    const M3 Rtr = mul(R1p, Rz);
    const double sin_g = -Rtr.m[0][1], cos_g = Rtr.m[1][1];
    const M3 Rg = rows3(v3(cos_g, -sin_g, 0), v3(sin_g, cos_g, 0), v3(0, 0, 1));
    const double t_initial = atan2(-Rtr.m[2][0], Rtr.m[2][2]);
    const M3 RzT = transpose(Rz);
    V3 pt[4];
    M3 Ft[4], avg = {};
    for (int i = 0; i < 4; i++) {
        pt[i] = mul(RzT, p[i]);
        Ft[i] = line_projector(mul(Rt, v[i]));
        for (int a = 0; a < 3; a++)
            for (int b = 0; b < 3; b++) avg.m[a][b] += Ft[i].m[a][b];
    }
    M3 G = identity();
    for (int a = 0; a < 3; a++)
        for (int b = 0; b < 3; b++) G.m[a][b] -= 0.25 * avg.m[a][b];
    G = inverse(G);
    for (int a = 0; a < 3; a++)
        for (int b = 0; b < 3; b++) G.m[a][b] *= 0.25;
    const M3 M1 = rows3(v3(0, 0, 2), v3(0, 0, 0), v3(-2, 0, 0));
    const M3 M2 = rows3(v3(-1, 0, 0), v3(0, 1, 0), v3(0, 0, -1));
    const M3 RgM1 = mul(Rg, M1), RgM2 = mul(Rg, M2);
    V3 b0 = v3(0, 0, 0), b1 = b0, b2 = b0;
    for (int i = 0; i < 4; i++) {
        const V3 x0 = mul(Rg, pt[i]), x1 = mul(RgM1, pt[i]), x2 = mul(RgM2, pt[i]);
        b0 = add(b0, sub(mul(Ft[i], x0), x0));
        b1 = add(b1, sub(mul(Ft[i], x1), x1));
        b2 = add(b2, sub(mul(Ft[i], x2), x2));
    }
    b0 = mul(G, b0), b1 = mul(G, b1), b2 = mul(G, b2);
    double a0 = 0, a1 = 0, a2 = 0, a3 = 0, a4 = 0;
    for (int i = 0; i < 4; i++) {
        const V3 y0 = add(mul(Rg, pt[i]), b0), y1 = add(mul(RgM1, pt[i]), b1), y2 = add(mul(RgM2, pt[i]), b2);
        const V3 c0 = sub(y0, mul(Ft[i], y0)), c1 = sub(y1, mul(Ft[i], y1)), c2 = sub(y2, mul(Ft[i], y2));
        a0 += dot(c0, c0);
        a1 += 2 * dot(c0, c1);
        a2 += dot(c1, c1) + 2 * dot(c0, c2);
        a3 += 2 * dot(c1, c2);
        a4 += dot(c2, c2);
    }
    const double poly[5] = {a1, 2 * a2 - 4 * a0, 3 * a3 - 3 * a1, 4 * a4 - 2 * a2, -a3};
    double roots[4];
    const int nr = PolyRoots<4>::solve(poly, roots);
    double minima[4];
    int nm = 0;
    for (int i = 0; i < nr; i++) {
        const double t1 = roots[i], t2 = t1 * t1, t3 = t1 * t2, t4 = t1 * t3, t5 = t1 * t4;
        if (a2 - 2 * a0 + (3 * a3 - 6 * a1) * t1 + (6 * a4 - 8 * a2 + 10 * a0) * t2 + (-8 * a3 + 6 * a1) * t3 +
                (-6 * a4 + 3 * a2) * t4 + a3 * t5 >= 0 &&
            fabs(2 * atan(roots[i]) - t_initial) > 0.1)
            minima[nm++] = roots[i];
    }
    if (nm != 1) return false;
    const double tc = minima[0];
    M3 Rb;
    for (int a = 0; a < 3; a++)
        for (int b = 0; b < 3; b++) Rb.m[a][b] = ((M2.m[a][b] * tc + M1.m[a][b]) * tc + I3.m[a][b]) / (1 + tc * tc);
    *out = mul(mul(mul(transpose(Rt), Rg), Rb), RzT);
    return true;
}

struct PoseInput {
    double H[9];
    double p[4][2];
};

__host__ __device__ inline void estimate(const PoseInput &d, double tagsize, double fx, double fy, double cx, double cy,
                                         int iters, at_pose *out) {
    const double s = tagsize / 2.0;
    const V3 p[4] = {v3(-s, s, 0), v3(s, s, 0), v3(s, -s, 0), v3(-s, -s, 0)};
    V3 v[4];
    for (int i = 0; i < 4; i++) v[i] = v3((d.p[i][0] - cx) / fx, (d.p[i][1] - cy) / fy, 1);
    M3 R1;
    V3 t1;
    homography_pose(d.H, s, fx, fy, cx, cy, &R1, &t1);
    const double e1 = orthogonal_iteration(v, p, &t1, &R1, iters);
    M3 R2;
    V3 t2 = v3(0, 0, 0);
    double e2 = HUGE_VAL;
    const bool two = second_minimum(v, p, t1, R1, &R2);
    if (two) e2 = orthogonal_iteration(v, p, &t2, &R2, iters);
    for (int a = 0; a < 3; a++)
        for (int b = 0; b < 3; b++) {
            out->R[3 * a + b] = R1.m[a][b];
            out->R2[3 * a + b] = two ? R2.m[a][b] : 0.0;
        }
    out->t[0] = t1.x, out->t[1] = t1.y, out->t[2] = t1.z;
    out->t2[0] = t2.x, out->t2[1] = t2.y, out->t2[2] = t2.z;
    out->err = e1;
    out->err2 = e2;
}

__global__ void k_pose(const PoseInput *in, int64_t n, double tagsize, double fx, double fy, double cx, double cy,
                       int iters, at_pose *out) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        estimate(in[i], tagsize, fx, fy, cx, cy, iters, out + i);
}

__global__ void k_homography_pose(const PoseInput *in, double tagsize, double fx, double fy, double cx, double cy,
                                  at_pose *out) {
    M3 R;
    V3 t;
    homography_pose(in->H, tagsize / 2.0, fx, fy, cx, cy, &R, &t);
    for (int a = 0; a < 9; a++) out->R[a] = R.m[a / 3][a % 3];
    out->t[0] = t.x, out->t[1] = t.y, out->t[2] = t.z;
    out->err = out->err2 = 0;
}

// One launch on the current device: n inputs to n poses (host arrays).
// mode 0: the full estimate (iters steps), 1: the homography pose only.
int run_poses(const PoseInput *in, int64_t n, double tagsize, double fx, double fy, double cx, double cy, int iters,
              int mode, at_pose *out) {
    if (n <= 0) return 0;
    PoseInput *d_in = nullptr;
    at_pose *d_out = nullptr;
    cudaStream_t st = nullptr;
    int rc = 0;
    if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) return 2;
    if (cudaMallocAsync((void **)&d_in, sizeof(PoseInput) * n, st) != cudaSuccess ||
        cudaMallocAsync((void **)&d_out, sizeof(at_pose) * n, st) != cudaSuccess) {
        rc = 2;
    } else {
        cudaMemcpyAsync(d_in, in, sizeof(PoseInput) * n, cudaMemcpyHostToDevice, st);
        if (mode == 0)
            k_pose<<<(unsigned)((n + 127) / 128), 128, 0, st>>>(d_in, n, tagsize, fx, fy, cx, cy, iters, d_out);
        else
            k_homography_pose<<<1, 1, 0, st>>>(d_in, tagsize, fx, fy, cx, cy, d_out);
        cudaMemcpyAsync(out, d_out, sizeof(at_pose) * n, cudaMemcpyDeviceToHost, st);
        if (cudaStreamSynchronize(st) != cudaSuccess || cudaGetLastError() != cudaSuccess) rc = 2;
    }
    if (d_in) cudaFreeAsync(d_in, st);
    if (d_out) cudaFreeAsync(d_out, st);
    cudaStreamSynchronize(st);
    cudaStreamDestroy(st);
    if (rc) fprintf(stderr, "apriltag_b200: pose estimation failed on the device\n");
    return rc;
}

PoseInput input_of(const double *H, const double (*p)[2]) {
    PoseInput d;
    memcpy(d.H, H, sizeof d.H);
    memcpy(d.p, p, sizeof d.p);
    return d;
}

matd_t *matd_from(const double *a, int rows, int cols) { return matd_create_data(rows, cols, a); }

}  // namespace

extern "C" {

int at_estimate_poses(const at_detector *td, double tagsize, double fx, double fy, double cx, double cy,
                      at_pose *out) {
    if (td == nullptr || out == nullptr) return 1;
    const int64_t n = td->ndetections;
    std::vector<PoseInput> in((size_t)(n > 0 ? n : 1));
    for (int64_t i = 0; i < n; i++) in[i] = input_of(td->detections[i].H, td->detections[i].p);
    return run_poses(in.data(), n, tagsize, fx, fy, cx, cy, 50, 0, out);
}

void estimate_pose_for_tag_homography(apriltag_detection_info_t *info, apriltag_pose_t *solution) {
    const PoseInput in = input_of(info->det->H->data, info->det->p);
    at_pose o;
    memset(&o, 0, sizeof o);
    run_poses(&in, 1, info->tagsize, info->fx, info->fy, info->cx, info->cy, 0, 1, &o);
    solution->R = matd_from(o.R, 3, 3);
    solution->t = matd_from(o.t, 3, 1);
}

void estimate_tag_pose_orthogonal_iteration(apriltag_detection_info_t *info, double *err1, apriltag_pose_t *pose1,
                                            double *err2, apriltag_pose_t *pose2, int nIters) {
    const PoseInput in = input_of(info->det->H->data, info->det->p);
    at_pose o;
    memset(&o, 0, sizeof o);
    run_poses(&in, 1, info->tagsize, info->fx, info->fy, info->cx, info->cy, nIters, 0, &o);
    pose1->R = matd_from(o.R, 3, 3);
    pose1->t = matd_from(o.t, 3, 1);
    *err1 = o.err;
    if (o.err2 != HUGE_VAL) {
        pose2->R = matd_from(o.R2, 3, 3);
        pose2->t = matd_from(o.t2, 3, 1);
    } else {
        pose2->R = nullptr;
        pose2->t = nullptr;
    }
    *err2 = o.err2;
}

double estimate_tag_pose(apriltag_detection_info_t *info, apriltag_pose_t *pose) {
    double e1, e2;
    apriltag_pose_t p1, p2;
    estimate_tag_pose_orthogonal_iteration(info, &e1, &p1, &e2, &p2, 50);
    if (e1 <= e2) {
        *pose = p1;
        matd_destroy(p2.R);
        matd_destroy(p2.t);
        return e1;
    }
    *pose = p2;
    matd_destroy(p1.R);
    matd_destroy(p1.t);
    return e2;
}

}  // extern "C"
