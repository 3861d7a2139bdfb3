// chain.cu: the source chain built on the device from the base plane (src/mips.cpp:80-84 over src/image.h:343-364).
//
// The default chain is the iterated 2x2 box: level i + 1 at (x, y) is 0.25 ((a + b) + (c + d)) of the four texels
// (2x, 2y), (2x + 1, 2y), (2x, 2y + 1), (2x + 1, 2y + 1) of level i, a missing second column or row (a one-wide or
// one-high level) repeating the only one there is, every channel on its own. The same float operations in the same
// order, so the same bits as the reference's host loop. One thread per output value; the levels in turn on the model's
// stream, so a caller uploads only the base plane.

#include "device.cuh"

namespace nb
{

__global__ void k_box(const float* in, int iw, int ih, float* out, int ow, int oh, int nc)
{
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (size_t)ow * oh * nc)
        return;
    const int k = (int)(i % (size_t)nc);
    const size_t p = i / (size_t)nc;
    const int x = (int)(p % (size_t)ow), y = (int)(p / (size_t)ow);
    const int xa = 2 * x < iw ? 2 * x : iw - 1, xb = 2 * x + 1 < iw ? 2 * x + 1 : iw - 1;
    const int ya = 2 * y < ih ? 2 * y : ih - 1, yb = 2 * y + 1 < ih ? 2 * y + 1 : ih - 1;
    const float a = in[((size_t)ya * iw + xa) * nc + k], b = in[((size_t)ya * iw + xb) * nc + k];
    const float c = in[((size_t)yb * iw + xa) * nc + k], d = in[((size_t)yb * iw + xb) * nc + k];
    out[i] = 0.25f * ((a + b) + (c + d));
}

int build_source_chain(nntc_b200_device* d)
{
    for (size_t i = 1; i < d->planes.size(); i++)
    {
        const DevPlane& a = d->planes[i - 1];
        const DevPlane& b = d->planes[i];
        const size_t n = (size_t)b.w0 * b.h0 * d->nout;
        k_box<<<grid_for(n, 256), 256, 0, d->stream>>>(a.src, a.w0, a.h0, b.src, b.w0, b.h0, d->nout);
        NB_LAUNCHED();
    }
    NB_CUDA(cudaStreamSynchronize(d->stream));
    return NNTC_B200_OK;
}

}   // namespace nb
