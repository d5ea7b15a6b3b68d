// Landmark term of the cost function (Plastimatch src/register/
// bspline_landmarks.cxx:25-134, bspline_landmarks_score_a): for each pair,
// the fixed landmark carried by the B-spline field, its squared distance to
// the moving landmark, and that distance's gradient spread over the 64
// knots of the landmark's tile.
//
// The reference evaluates this term in float, one landmark after another.
// The device keeps its arithmetic: every product and sum is rounded to
// float in the reference's order (no contraction into FMA), so score and
// gradient match the reference bit for bit.
//   kernel 1  one thread per landmark: field at the landmark (the 64 q_lut
//             weights in the reference's slot order), residual, dc/dv;
//   kernel 2  one thread per knot: the contributions of every landmark
//             whose tile touches the knot, added in landmark order (the
//             order the reference adds them in), plus the score: the
//             squared distances summed in landmark order by one thread.
#include "kernels.cuh"

namespace b200 {

// p[3l..3l+2]: the landmark's tile; w[64l + m]: its q_lut row (slot m =
// i + 4j + 16k); fm[6l]: fixed xyz then moving xyz.  Writes dc[4l..4l+3]:
// dc/dv xyz and the squared distance.
__global__ void
landmark_residual_kernel (int n, const int* __restrict__ p,
    const float* __restrict__ w, const float* __restrict__ fm,
    const float* __restrict__ coeff, int cd0, int cd1, float grad_coeff,
    float* __restrict__ dc)
{
    const int l = blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= n) return;
    const int px = p[3 * l], py = p[3 * l + 1], pz = p[3 * l + 2];
    const float* wl = w + 64 * (size_t) l;
    // bspline_interp_pix (src/base/bspline_interpolate.cxx:21-48)
    float d0 = 0.f, d1 = 0.f, d2 = 0.f;
    int m = 0;
    for (int k = 0; k < 4; k++) {
        for (int j = 0; j < 4; j++) {
            for (int i = 0; i < 4; i++) {
                const size_t cidx = 3 * ((size_t) (pz + k) * cd1 * cd0
                    + (size_t) (py + j) * cd0 + (px + i));
                const float q = wl[m];
                d0 = __fadd_rn (d0, __fmul_rn (q, coeff[cidx + 0]));
                d1 = __fadd_rn (d1, __fmul_rn (q, coeff[cidx + 1]));
                d2 = __fadd_rn (d2, __fmul_rn (q, coeff[cidx + 2]));
                m++;
            }
        }
    }
    const float* f = fm + 6 * (size_t) l;
    const float e0 = __fsub_rn (f[3], __fadd_rn (f[0], d0));
    const float e1 = __fsub_rn (f[4], __fadd_rn (f[1], d1));
    const float e2 = __fsub_rn (f[5], __fadd_rn (f[2], d2));
    const float dist = __fadd_rn (__fadd_rn (__fmul_rn (e0, e0),
        __fmul_rn (e1, e1)), __fmul_rn (e2, e2));
    float* o = dc + 4 * (size_t) l;
    o[0] = __fmul_rn (-grad_coeff, e0);
    o[1] = __fmul_rn (-grad_coeff, e1);
    o[2] = __fmul_rn (-grad_coeff, e2);
    o[3] = dist;
}

// Adds the landmark gradient into grad (xyz interleaved per knot) and
// writes lmetric = (sum of squared distances) / n.
__global__ void
landmark_grad_kernel (int n, const int* __restrict__ p,
    const float* __restrict__ w, const float* __restrict__ dc, int cd0,
    int cd1, int cd2, float* __restrict__ grad, float* __restrict__ lmetric)
{
    const long long nk = (long long) cd0 * cd1 * cd2;
    const long long c = (long long) blockIdx.x * blockDim.x + threadIdx.x;
    if (c == 0) {
        // land_score accumulated in landmark order, then divided by n
        float s = 0.f;
        for (int l = 0; l < n; l++) s = __fadd_rn (s, dc[4 * l + 3]);
        *lmetric = __fdiv_rn (s, (float) n);
    }
    if (c >= nk) return;
    const int kx = (int) (c % cd0);
    const int ky = (int) ((c / cd0) % cd1);
    const int kz = (int) (c / ((long long) cd0 * cd1));
    float g0 = 0.f, g1 = 0.f, g2 = 0.f;
    bool touched = false;
    for (int l = 0; l < n; l++) {
        const unsigned i = (unsigned) (kx - p[3 * l]);
        const unsigned j = (unsigned) (ky - p[3 * l + 1]);
        const unsigned k = (unsigned) (kz - p[3 * l + 2]);
        if (i > 3u || j > 3u || k > 3u) continue;
        if (!touched) {
            g0 = grad[3 * c + 0];
            g1 = grad[3 * c + 1];
            g2 = grad[3 * c + 2];
            touched = true;
        }
        // Bspline_score::update_grad (src/register/bspline_score.cxx:
        // 117-143): grad += dc_dv * q_lut[m]
        const float q = w[64 * (size_t) l + i + 4 * j + 16 * k];
        g0 = __fadd_rn (g0, __fmul_rn (dc[4 * l + 0], q));
        g1 = __fadd_rn (g1, __fmul_rn (dc[4 * l + 1], q));
        g2 = __fadd_rn (g2, __fmul_rn (dc[4 * l + 2], q));
    }
    if (touched) {
        grad[3 * c + 0] = g0;
        grad[3 * c + 1] = g1;
        grad[3 * c + 2] = g2;
    }
}

cudaError_t
launch_landmarks (const BspGeom& g, int n, const int* p, const float* w,
    const float* fm, const float* coeff, float grad_coeff, float* dc,
    float* grad, float* lmetric, cudaStream_t st)
{
    if (n < 1) return cudaErrorInvalidValue;
    landmark_residual_kernel<<<(n + 127) / 128, 128, 0, st>>> (n, p, w, fm,
        coeff, g.cdims[0], g.cdims[1], grad_coeff, dc);
    const long long nk = (long long) g.cdims[0] * g.cdims[1] * g.cdims[2];
    landmark_grad_kernel<<<(unsigned) ((nk + 255) / 256), 256, 0, st>>> (n, p,
        w, dc, g.cdims[0], g.cdims[1], g.cdims[2], grad, lmetric);
    return cudaGetLastError ();
}

} // namespace b200
