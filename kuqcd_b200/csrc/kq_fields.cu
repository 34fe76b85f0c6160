// Field layout conversion and synthetic field generation on the device.
//
// Host records (the reference's NORMAL_ORDER layout, kuqcd.cpp:103-169, one rank):
//   gauge  rec[reim + 2*(l + 9*(dir + 4*s))], s in [0, V): even sites (s = i_cb) then odd sites (s = Vh + i_cb)
//   spinor rec[reim + 2*(c + 3*i_cb)] over one parity
// BATCH_ORDER records (kuqcd.cpp:112-124, latt_base.cpp:77-93) are reordered to NORMAL_ORDER on the host side
// before they reach these kernels (kq_capi.cu).
#include "kq_dslash_core.cuh"

namespace kq {

Geom make_geom(const unsigned lat[4])
{
    Geom g;
    for (int i = 0; i < 4; ++i) g.n[i] = (int)lat[i];
    g.hx = g.n[0] / 2;
    g.vh = (int)((size_t)lat[0] * lat[1] * lat[2] * lat[3] / 2);
    g.sy = g.hx;
    g.sz = g.hx * g.n[1];
    g.st = g.hx * g.n[1] * g.n[2];
    return g;
}

size_t spinor_bytes(const Geom &g, int prec)
{
    const size_t pv = (size_t)pad_sites(g.vh);
    return prec == P64 ? 48 * pv : prec == P32 ? 24 * pv : 16 * pv;
}

size_t links_bytes(const Geom &g, int prec)
{
    const size_t pv = (size_t)pad_sites(g.vh);
    return 4 * pv * (prec == P64 ? 144 : prec == P32 ? 72 : 36);
}

// ------------------------------------------------------------------------------------------------ links
template <typename R>
__global__ void rec_absmax_kernel(const R *__restrict__ rec, size_t n, unsigned *out)
{
    float m = 0.f;
    for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x)
        m = fmaxf(m, fabsf((float)rec[k]));
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_down_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) atomicMax(out, __float_as_uint(m));  // non-negative floats order as integers
}

template <int OP, typename R>
__global__ void links_from_rec_kernel(Geom g, int pv, const R *__restrict__ rec, double factor, float scale,
                                      void *out0, void *out1)
{
    const int V = 2 * g.vh;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 4 * V) return;
    const int s = t >> 2, dir = t & 3;
    const int par = s >= g.vh ? 1 : 0;
    const int i = s - par * g.vh;
    double u[18];
    const R *r = rec + (size_t)18 * (dir + 4 * (size_t)s);
#pragma unroll
    for (int k = 0; k < 18; ++k) u[k] = factor * (double)r[k];
    st_link<OP>(par ? out1 : out0, pv, dir, i, scale, u);
}

template <int IP, int OP>
__global__ void links_convert_kernel(Geom g, int pv, LinkSet in, LinkSet out)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 8 * g.vh) return;
    const int par = t / (4 * g.vh);
    const int rem = t - par * 4 * g.vh;
    const int dir = rem / g.vh, i = rem - dir * g.vh;
    typename Acc<IP>::T u[18];
    ld_link_any<IP>(in.par[par], pv, dir, i, in.scale, in.recon, u);
    double d[18];
#pragma unroll
    for (int k = 0; k < 18; ++k) d[k] = (double)u[k];
    st_link<OP>(out.par[par], pv, dir, i, out.scale, d);
}

template <int IP>
__global__ void links_absmax_kernel(Geom g, int pv, LinkSet in, unsigned *out)
{
    float m = 0.f;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < 8 * g.vh; t += gridDim.x * blockDim.x) {
        const int par = t / (4 * g.vh);
        const int rem = t - par * 4 * g.vh;
        const int dir = rem / g.vh, i = rem - dir * g.vh;
        typename Acc<IP>::T u[18];
        ld_link_any<IP>(in.par[par], pv, dir, i, in.scale, in.recon, u);
#pragma unroll
        for (int k = 0; k < 18; ++k) m = fmaxf(m, fabsf((float)u[k]));
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_down_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) atomicMax(out, __float_as_uint(m));
}

cudaError_t links_from_host_record(const Geom &g, const void *d_rec, int rec_prec, double factor, LinkSet &out,
                                   int out_prec, unsigned *m, cudaStream_t s)
{
    const int pv = pad_sites(g.vh);
    const size_t n = (size_t)2 * g.vh * 72;
    out.scale = 1.f;
    out.recon = 0;
    if (out_prec == P16) {
        KQ_CUDA_TRY(cudaMemsetAsync(m, 0, sizeof(unsigned), s));
        if (rec_prec == P64)
            rec_absmax_kernel<double><<<592, 256, 0, s>>>(static_cast<const double *>(d_rec), n, m);
        else
            rec_absmax_kernel<float><<<592, 256, 0, s>>>(static_cast<const float *>(d_rec), n, m);
        unsigned h = 0;
        KQ_CUDA_TRY(cudaMemcpyAsync(&h, m, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
        KQ_CUDA_TRY(cudaStreamSynchronize(s));
        float am;
        memcpy(&am, &h, sizeof(float));
        out.scale = (float)(am * fabs(factor));
        if (out.scale == 0.f) out.scale = 1.f;
    }
    const int threads = 256, blocks = (8 * g.vh + threads - 1) / threads;
#define KQ_L(OP)                                                                                          \
    if (rec_prec == P64)                                                                                  \
        links_from_rec_kernel<OP, double><<<blocks, threads, 0, s>>>(g, pv, static_cast<const double *>(d_rec), \
                                                                     factor, out.scale, out.par[0], out.par[1]); \
    else                                                                                                  \
        links_from_rec_kernel<OP, float><<<blocks, threads, 0, s>>>(g, pv, static_cast<const float *>(d_rec), \
                                                                    factor, out.scale, out.par[0], out.par[1]);
    switch (out_prec) {
        case P64: KQ_L(0); break;
        case P32: KQ_L(1); break;
        default: KQ_L(2); break;
    }
#undef KQ_L
    return cudaGetLastError();
}

float links_absmax(const Geom &g, const LinkSet &in, int in_prec, unsigned *m, cudaStream_t s)
{
    cudaMemsetAsync(m, 0, sizeof(unsigned), s);
    const int pv = pad_sites(g.vh);
    switch (in_prec) {
        case P64: links_absmax_kernel<0><<<592, 256, 0, s>>>(g, pv, in, m); break;
        case P32: links_absmax_kernel<1><<<592, 256, 0, s>>>(g, pv, in, m); break;
        default: links_absmax_kernel<2><<<592, 256, 0, s>>>(g, pv, in, m); break;
    }
    unsigned h = 0;
    cudaMemcpyAsync(&h, m, sizeof(unsigned), cudaMemcpyDeviceToHost, s);
    if (cudaStreamSynchronize(s) != cudaSuccess) return -1.f;
    float am;
    memcpy(&am, &h, sizeof(float));
    return am;
}

cudaError_t links_convert(const Geom &g, const LinkSet &in, int in_prec, LinkSet &out, int out_prec, unsigned *m,
                          cudaStream_t s)
{
    const int pv = pad_sites(g.vh);
    out.scale = 1.f;
    out.recon = 0;
    if (out_prec == P16) {
        const float am = links_absmax(g, in, in_prec, m, s);
        if (am < 0.f) {
            set_last_error("links_convert: absmax failed");
            return cudaErrorUnknown;
        }
        out.scale = am > 0.f ? am : 1.f;
    }
    const int threads = 256, blocks = (8 * g.vh + threads - 1) / threads;
#define KQ_C(IP, OP) links_convert_kernel<IP, OP><<<blocks, threads, 0, s>>>(g, pv, in, out)
    if (in_prec == P64 && out_prec == P32) KQ_C(0, 1);
    else if (in_prec == P64 && out_prec == P16) KQ_C(0, 2);
    else if (in_prec == P32 && out_prec == P16) KQ_C(1, 2);
    else if (in_prec == P32 && out_prec == P64) KQ_C(1, 0);
    else if (in_prec == P64 && out_prec == P64) KQ_C(0, 0);
    else if (in_prec == P32 && out_prec == P32) KQ_C(1, 1);
    else {
        set_last_error("links_convert: unsupported precision pair");
        return cudaErrorInvalidValue;
    }
#undef KQ_C
    return cudaGetLastError();
}

// ------------------------------------------------------------------------------------------------ compression
// A link L = s W with W in SU(3) and s real has det L = s^3 and row 2 = conj(row0 x row1) / s.  The check kernel
// returns the largest |row2 - conj(row0 x row1) / s| / |s| (or a huge value where det L is not real and nonzero);
// the pack kernel writes rows 0 and 1 and 1/s in the compressed layout of kq_prec.cuh.
__device__ __forceinline__ double link_scale_from_det(const double u[18], double *det_im)
{
    // det = sum_c row0_c * (row1 x row2)_c
    double dr = 0.0, di = 0.0;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        const int c1 = (c + 1) % 3, c2 = (c + 2) % 3;
        const double xr = (u[6 + 2 * c1] * u[12 + 2 * c2] - u[6 + 2 * c1 + 1] * u[12 + 2 * c2 + 1]) -
                          (u[6 + 2 * c2] * u[12 + 2 * c1] - u[6 + 2 * c2 + 1] * u[12 + 2 * c1 + 1]);
        const double xi = (u[6 + 2 * c1] * u[12 + 2 * c2 + 1] + u[6 + 2 * c1 + 1] * u[12 + 2 * c2]) -
                          (u[6 + 2 * c2] * u[12 + 2 * c1 + 1] + u[6 + 2 * c2 + 1] * u[12 + 2 * c1]);
        dr += u[2 * c] * xr - u[2 * c + 1] * xi;
        di += u[2 * c] * xi + u[2 * c + 1] * xr;
    }
    *det_im = di;
    return cbrt(dr);
}

template <int IP>
__global__ void links_recon_check_kernel(Geom g, int pv, LinkSet in, double tol, unsigned *out)
{
    float m = 0.f;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < 8 * g.vh; t += gridDim.x * blockDim.x) {
        const int par = t / (4 * g.vh);
        const int rem = t - par * 4 * g.vh;
        const int dir = rem / g.vh, i = rem - dir * g.vh;
        typename Acc<IP>::T uf[18];
        ld_link<IP>(par ? in.par[1] : in.par[0], pv, dir, i, in.scale, uf);
        double u[18], w[18];
#pragma unroll
        for (int k = 0; k < 18; ++k) w[k] = u[k] = (double)uf[k];
        double di;
        const double sc = link_scale_from_det(u, &di);
        float err = 3.0e38f;
        if (sc != 0.0 && fabs(di) <= tol * fabs(sc * sc * sc)) {
            rebuild_row2(w, 1.0 / sc);
            double e = 0.0;
#pragma unroll
            for (int k = 12; k < 18; ++k) e = fmax(e, fabs(w[k] - u[k]));
            err = (float)(e / fabs(sc));
        }
        m = fmaxf(m, err);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_down_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) atomicMax(out, __float_as_uint(m));
}

template <int IP>
__global__ void links_recon_pack_kernel(Geom g, int pv, LinkSet in, void *out0, void *out1)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 8 * g.vh) return;
    const int par = t / (4 * g.vh);
    const int rem = t - par * 4 * g.vh;
    const int dir = rem / g.vh, i = rem - dir * g.vh;
    typename Acc<IP>::T uf[18];
    ld_link<IP>(par ? in.par[1] : in.par[0], pv, dir, i, in.scale, uf);
    double u[18];
#pragma unroll
    for (int k = 0; k < 18; ++k) u[k] = (double)uf[k];
    double di;
    const double sc = link_scale_from_det(u, &di);
    st_link_recon<IP>(par ? out1 : out0, pv, dir, i, u, 1.0 / sc);
}

// Compress a full-storage FP64 or FP32 link set in place when every link passes the check (relative
// reconstruction error below tol); *done reports whether it did.
cudaError_t links_compress(const Geom &g, LinkSet &lk, int prec, double tol, unsigned *m, cudaStream_t s, bool *done)
{
    *done = false;
    if ((prec != P64 && prec != P32) || lk.recon) return cudaSuccess;
    const int pv = pad_sites(g.vh);
    KQ_CUDA_TRY(cudaMemsetAsync(m, 0, sizeof(unsigned), s));
    if (prec == P64) links_recon_check_kernel<0><<<592, 256, 0, s>>>(g, pv, lk, tol, m);
    else links_recon_check_kernel<1><<<592, 256, 0, s>>>(g, pv, lk, tol, m);
    KQ_CUDA_TRY(cudaGetLastError());
    unsigned h = 0;
    KQ_CUDA_TRY(cudaMemcpyAsync(&h, m, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
    KQ_CUDA_TRY(cudaStreamSynchronize(s));
    float err;
    memcpy(&err, &h, sizeof(float));
    if (!(err <= tol)) return cudaSuccess;
    const size_t part = (size_t)(prec == P64 ? 104 : 52) * 4 * pv;  // one parity, 4 directions
    void *tmp = nullptr;
    KQ_CUDA_TRY(cudaMallocAsync(&tmp, 2 * part, s));
    char *t0 = static_cast<char *>(tmp);
    const int threads = 256, blocks = (8 * g.vh + threads - 1) / threads;
    if (prec == P64) links_recon_pack_kernel<0><<<blocks, threads, 0, s>>>(g, pv, lk, t0, t0 + part);
    else links_recon_pack_kernel<1><<<blocks, threads, 0, s>>>(g, pv, lk, t0, t0 + part);
    cudaError_t e = cudaGetLastError();
    // the compressed parity fields fit in the full-storage regions they replace
    if (e == cudaSuccess) e = cudaMemcpyAsync(lk.par[0], t0, part, cudaMemcpyDeviceToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(lk.par[1], t0 + part, part, cudaMemcpyDeviceToDevice, s);
    cudaFreeAsync(tmp, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    KQ_CUDA_TRY(e);
    lk.recon = 1;
    *done = true;
    return cudaSuccess;
}

// ------------------------------------------------------------------------------------------------ spinors
template <int P, typename R>
__global__ void spinor_from_rec_kernel(Geom g, int pv, const R *__restrict__ rec, void *dst)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= g.vh) return;
    typename Acc<P>::T v[6];
#pragma unroll
    for (int k = 0; k < 6; ++k) v[k] = (typename Acc<P>::T)rec[6 * (size_t)i + k];
    st_spinor<P>(dst, pv, i, v);
}

template <int P, typename R>
__global__ void spinor_to_rec_kernel(Geom g, int pv, const void *src, R *__restrict__ rec)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= g.vh) return;
    typename Acc<P>::T v[6];
    ld_spinor<P>(src, pv, i, v);
#pragma unroll
    for (int k = 0; k < 6; ++k) rec[6 * (size_t)i + k] = (R)v[k];
}

template <int IP, int OP>
__global__ void spinor_convert_kernel(Geom g, int pv, const void *src, void *dst)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= g.vh) return;
    typename Acc<IP>::T v[6];
    ld_spinor<IP>(src, pv, i, v);
    typename Acc<OP>::T w[6];
#pragma unroll
    for (int k = 0; k < 6; ++k) w[k] = (typename Acc<OP>::T)v[k];
    st_spinor<OP>(dst, pv, i, w);
}

cudaError_t spinor_from_record(const Geom &g, const void *d_rec, int rec_prec, void *dst, int prec, cudaStream_t s)
{
    const int pv = pad_sites(g.vh), bs = 256, nb = (g.vh + bs - 1) / bs;
#define KQ_S(P)                                                                                                      \
    if (rec_prec == P64)                                                                                             \
        spinor_from_rec_kernel<P, double><<<nb, bs, 0, s>>>(g, pv, static_cast<const double *>(d_rec), dst);        \
    else                                                                                                             \
        spinor_from_rec_kernel<P, float><<<nb, bs, 0, s>>>(g, pv, static_cast<const float *>(d_rec), dst);
    switch (prec) {
        case P64: KQ_S(0); break;
        case P32: KQ_S(1); break;
        default: KQ_S(2); break;
    }
#undef KQ_S
    return cudaGetLastError();
}

cudaError_t spinor_to_record(const Geom &g, const void *src, int prec, void *d_rec, int rec_prec, cudaStream_t s)
{
    const int pv = pad_sites(g.vh), bs = 256, nb = (g.vh + bs - 1) / bs;
#define KQ_S(P)                                                                                                \
    if (rec_prec == P64)                                                                                       \
        spinor_to_rec_kernel<P, double><<<nb, bs, 0, s>>>(g, pv, src, static_cast<double *>(d_rec));          \
    else                                                                                                       \
        spinor_to_rec_kernel<P, float><<<nb, bs, 0, s>>>(g, pv, src, static_cast<float *>(d_rec));
    switch (prec) {
        case P64: KQ_S(0); break;
        case P32: KQ_S(1); break;
        default: KQ_S(2); break;
    }
#undef KQ_S
    return cudaGetLastError();
}

cudaError_t spinor_convert(const Geom &g, const void *src, int src_prec, void *dst, int dst_prec, cudaStream_t s)
{
    const int pv = pad_sites(g.vh), bs = 256, nb = (g.vh + bs - 1) / bs;
#define KQ_C(IP, OP) spinor_convert_kernel<IP, OP><<<nb, bs, 0, s>>>(g, pv, src, dst)
    if (src_prec == P64 && dst_prec == P32) KQ_C(0, 1);
    else if (src_prec == P64 && dst_prec == P16) KQ_C(0, 2);
    else if (src_prec == P32 && dst_prec == P64) KQ_C(1, 0);
    else if (src_prec == P16 && dst_prec == P64) KQ_C(2, 0);
    else if (src_prec == P32 && dst_prec == P16) KQ_C(1, 2);
    else if (src_prec == P16 && dst_prec == P32) KQ_C(2, 1);
    else if (src_prec == dst_prec) {
        return cudaMemcpyAsync(dst, src, spinor_bytes(g, src_prec), cudaMemcpyDeviceToDevice, s);
    }
#undef KQ_C
    return cudaGetLastError();
}

// ------------------------------------------------------------------------------------------------ generators
// Synthetic gauge and source fields: thin U_mu(x) = exp(i eps H) with H traceless Hermitian from seeded Gaussians,
// staggered phases eta folded in, fat = 9/8 eta U, long = -1/24 eta U(x) U(x+mu) U(x+2mu); Gaussian sources.
// A counter-based hash of (seed, counter) makes every value independent of launch shape.
__device__ __forceinline__ uint64_t gen_hash(uint64_t seed, uint64_t counter)
{
    uint64_t z = seed + 0x9E3779B97F4A7C15ull * (counter + 1);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z = z ^ (z >> 31);
    z += seed ^ 0xD1B54A32D192ED03ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

__device__ __forceinline__ double gen_unif(uint64_t seed, uint64_t c)
{
    return (double)((gen_hash(seed, c) >> 11) + 1) * (1.0 / 9007199254740992.0);
}

__device__ __forceinline__ void gen_gauss2(uint64_t seed, uint64_t k, double &a, double &b)
{
    const double u1 = gen_unif(seed, 2 * k), u2 = gen_unif(seed, 2 * k + 1);
    const double rad = sqrt(-2.0 * log(u1));
    double sn, cs;
    sincos(6.283185307179586476925 * u2, &sn, &cs);
    a = rad * cs;
    b = rad * sn;
}

__device__ __forceinline__ void cmul33(const double *A, const double *B, double *C)
{
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            double re = 0, im = 0;
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                const double ar = A[2 * (k + 3 * r)], ai = A[2 * (k + 3 * r) + 1];
                const double br = B[2 * (c + 3 * k)], bi = B[2 * (c + 3 * k) + 1];
                re += ar * br - ai * bi;
                im += ar * bi + ai * br;
            }
            C[2 * (c + 3 * r)] = re;
            C[2 * (c + 3 * r) + 1] = im;
        }
}

// exp(i eps H): scaling and squaring of a degree-16 Taylor polynomial (Horner form)
__device__ void gen_thin(uint64_t seed, uint64_t link, double eps, double *U)
{
    double A[18], X[18];
#pragma unroll
    for (int k = 0; k < 9; ++k) gen_gauss2(seed, 9 * link + k, A[2 * k], A[2 * k + 1]);
    double H[18];
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            H[2 * (c + 3 * r)] = 0.5 * (A[2 * (c + 3 * r)] + A[2 * (r + 3 * c)]);
            H[2 * (c + 3 * r) + 1] = 0.5 * (A[2 * (c + 3 * r) + 1] - A[2 * (r + 3 * c) + 1]);
        }
    const double tr = (H[0] + H[8] + H[16]) / 3.0;
    H[0] -= tr;
    H[8] -= tr;
    H[16] -= tr;
    double nrm = 0;
#pragma unroll
    for (int l = 0; l < 9; ++l) {
        X[2 * l] = -eps * H[2 * l + 1];
        X[2 * l + 1] = eps * H[2 * l];
        nrm += X[2 * l] * X[2 * l] + X[2 * l + 1] * X[2 * l + 1];
    }
    nrm = sqrt(nrm);
    int sq = 0;
    while (nrm > 0.25) {
        nrm *= 0.5;
        ++sq;
    }
    const double scale = ldexp(1.0, -sq);
#pragma unroll
    for (int l = 0; l < 18; ++l) X[l] *= scale;
    double P[18], T[18];
#pragma unroll
    for (int l = 0; l < 18; ++l) P[l] = 0.0;
    P[0] = P[8] = P[16] = 1.0;
    for (int k = 16; k >= 1; --k) {
        cmul33(X, P, T);
#pragma unroll
        for (int l = 0; l < 18; ++l) P[l] = T[l] / (double)k;
        P[0] += 1.0;
        P[8] += 1.0;
        P[16] += 1.0;
    }
    for (int s = 0; s < sq; ++s) {
        cmul33(P, P, T);
#pragma unroll
        for (int l = 0; l < 18; ++l) P[l] = T[l];
    }
#pragma unroll
    for (int l = 0; l < 18; ++l) U[l] = P[l];
}

__global__ void make_links_kernel(Geom g, double eps, uint64_t seed, double *fat, double *lng)
{
    const long V = 2L * g.vh;
    const long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (t >= 4 * V) return;
    const long lex = t >> 2;
    const int mu = (int)(t & 3);
    int c[4];
    long r = lex;
    c[0] = (int)(r % g.n[0]);
    r /= g.n[0];
    c[1] = (int)(r % g.n[1]);
    r /= g.n[1];
    c[2] = (int)(r % g.n[2]);
    c[3] = (int)(r / g.n[2]);
    const int par = (c[0] + c[1] + c[2] + c[3]) & 1;
    const long site = (long)(c[0] >> 1) + (long)g.hx * (c[1] + (long)g.n[1] * (c[2] + (long)g.n[2] * c[3])) +
                      (par ? g.vh : 0);
    auto lexof = [&](const int *cc) {
        return (uint64_t)cc[0] + (uint64_t)g.n[0] * (cc[1] + (uint64_t)g.n[1] * (cc[2] + (uint64_t)g.n[2] * cc[3]));
    };
    double U0[18], U1[18], U2[18], T[18], L[18];
    gen_thin(seed, 4 * lexof(c) + mu, eps, U0);
    int c1[4] = {c[0], c[1], c[2], c[3]}, c2[4] = {c[0], c[1], c[2], c[3]};
    c1[mu] = (c[mu] + 1) % g.n[mu];
    c2[mu] = (c[mu] + 2) % g.n[mu];
    gen_thin(seed, 4 * lexof(c1) + mu, eps, U1);
    gen_thin(seed, 4 * lexof(c2) + mu, eps, U2);
    cmul33(U0, U1, T);
    cmul33(T, U2, L);
    int ssum = 0;
    for (int k = 0; k < mu; ++k) ssum += c[k];
    const double e = (ssum & 1) ? -1.0 : 1.0;
    double *F = fat + 18 * (mu + 4 * site);
    double *N = lng + 18 * (mu + 4 * site);
#pragma unroll
    for (int l = 0; l < 18; ++l) {
        F[l] = (9.0 / 8.0) * e * U0[l];
        N[l] = (-1.0 / 24.0) * e * L[l];
    }
}

__global__ void make_source_kernel(Geom g, int parity, uint64_t seed, double *b)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= g.vh) return;
    const SiteCoord c = site_coord(g, i, parity);
    const uint64_t sseed = seed ^ 0x50C3A1E5D00DF00Dull;
    const uint64_t lex =
        (uint64_t)c.x + (uint64_t)g.n[0] * (c.y + (uint64_t)g.n[1] * (c.z + (uint64_t)g.n[2] * c.t));
#pragma unroll
    for (int k = 0; k < 3; ++k) gen_gauss2(sseed, 3 * lex + k, b[6 * (size_t)i + 2 * k], b[6 * (size_t)i + 2 * k + 1]);
}

cudaError_t make_links_record(const Geom &g, double eps, uint64_t seed, double *d_fat_rec, double *d_long_rec,
                              cudaStream_t s)
{
    const long n = 8L * g.vh;
    const int bs = 128;
    make_links_kernel<<<(unsigned)((n + bs - 1) / bs), bs, 0, s>>>(g, eps, seed, d_fat_rec, d_long_rec);
    return cudaGetLastError();
}

cudaError_t make_source_record(const Geom &g, int parity, uint64_t seed, double *d_rec, cudaStream_t s)
{
    const int bs = 256;
    make_source_kernel<<<(g.vh + bs - 1) / bs, bs, 0, s>>>(g, parity, seed, d_rec);
    return cudaGetLastError();
}

}  // namespace kq
