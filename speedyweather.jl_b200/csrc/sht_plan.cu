// libsht host side: the plan (precomputed tables, computed once in FP64 on the
// host and rounded once), argument checking, and the C ABI of include/sht.h.
//
// Replaces the SpectralTransform constructor, SpeedyTransforms/src/spectral_transform.jl:118-302,
// and the transform!/operator entry points (spectral_transform.jl:515-631,
// spectral_gradients.jl).
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <algorithm>
#include <new>
#include <thread>

#include "sht_internal.h"

namespace sht {
cudaError_t fft_set_smem(int bytes);
cudaError_t tc_prepare(Plan& p);       // tensor-core Legendre tables (sht_legendre_tc.cu)
void tc_release(Plan& p);
int tc_supported();
cudaError_t launch_legendre_synthesis_tc(const Plan& p, const float2* coeffs, int64_t ldc, int K, cudaStream_t s);
cudaError_t launch_legendre_analysis_tc(const Plan& p, float2* coeffs, int64_t ldc, int K, bool add, cudaStream_t s);
}  // namespace sht

using namespace sht;

// Host-buffer transforms (sht_synthesize_host / sht_analyze_host): device staging slots
// for chunks of layers, the plan's copy streams and the events ordering them.
struct HostPipe {
    int chunk = 0;                            // layers per chunk
    float2* in_slot[2] = {};                  // [chunk][nlm] coefficients on their way in
    float2* out_slot[2] = {};                 // [chunk][nlm] coefficients on their way out
    cudaStream_t copy_in = nullptr, copy_out = nullptr;
    cudaEvent_t in_ready[2] = {}, in_free[2] = {}, out_ready[2] = {}, out_free[2] = {};
    int in_next = 0, out_next = 0;            // slot used by the next chunk
};

struct sht_plan {
    Plan p;
    HostPipe host;
};

namespace {

thread_local std::string g_last_error;

int fail(int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return code;
}

int cuda_fail(cudaError_t e, const char* where) {
    if (e == cudaErrorMemoryAllocation) return fail(SHT_ENOMEM, "%s: %s", where, cudaGetErrorString(e));
    return fail(SHT_ECUDA, "%s: %s", where, cudaGetErrorString(e));
}

// n-point Gauss-Legendre nodes (ascending) and weights in FP64: Newton iteration on
// P_n (restates FastGaussQuadrature.gausslegendre, RingGrids/src/quadrature_weights.jl:11).
void gauss_legendre(int n, std::vector<double>& x, std::vector<double>& w) {
    x.assign(n, 0.0);
    w.assign(n, 0.0);
    const int half = (n + 1) / 2;
    for (int i = 0; i < half; ++i) {
        double z = std::cos(M_PI * (i + 0.75) / (n + 0.5));
        double dp = 1.0;
        for (int it = 0; it < 100; ++it) {
            double p0 = 1.0, p1 = z;
            for (int k = 2; k <= n; ++k) {
                const double p2 = ((2.0 * k - 1.0) * z * p1 - (k - 1.0) * p0) / k;
                p0 = p1;
                p1 = p2;
            }
            dp = n * (z * p1 - p0) / (z * z - 1.0);
            const double dz = p1 / dp;
            z -= dz;
            if (std::fabs(dz) < 1e-16) break;
        }
        double p0 = 1.0, p1 = z;
        for (int k = 2; k <= n; ++k) {
            const double p2 = ((2.0 * k - 1.0) * z * p1 - (k - 1.0) * p0) / k;
            p0 = p1;
            p1 = p2;
        }
        dp = n * (z * p1 - p0) / (z * z - 1.0);
        const double wt = 2.0 / ((1.0 - z * z) * dp * dp);
        // z is descending from ~1; store ascending
        x[n - 1 - i] = z;
        w[n - 1 - i] = wt;
        x[i] = -z;
        w[i] = wt;
    }
    if (n % 2 == 1) x[n / 2] = 0.0;
}

// Prime factorisation into Stockham radices, in stage order: primes above 8 first
// (largest first; the first stage needs no twiddles), then 7, 5, 3, then the power of
// two as radix-8 stages with one radix-4 or radix-2 (or two radix-4) for the rest.
int factorize(int n, int32_t* fac) {
    std::vector<int> f;
    int m = n;
    for (int p = 2; (int64_t)p * p <= m; ++p)
        while (m % p == 0) {
            f.push_back(p);
            m /= p;
        }
    if (m > 1) f.push_back(m);
    std::vector<int> out;
    for (auto it = f.rbegin(); it != f.rend(); ++it)
        if (*it > 8) out.push_back(*it);
    for (int q : {7, 5, 3})
        for (int x : f)
            if (x == q) out.push_back(q);
    int twos = (int)std::count(f.begin(), f.end(), 2);
    if (twos % 3 == 1 && twos >= 4) {
        out.push_back(4);
        out.push_back(4);
        twos -= 4;
    }
    for (; twos >= 3; twos -= 3) out.push_back(8);
    if (twos == 2) out.push_back(4);
    if (twos == 1) out.push_back(2);
    if ((int)out.size() > kMaxFactors) return -1;
    for (size_t i = 0; i < out.size(); ++i) fac[i] = out[i];
    return (int)out.size();
}

// FFT cost of one layer of a ring: FMAs of the prime stages (2 n hpad each) plus ~3 n per
// small-radix stage and ~4 n of copies; with pre, the first (prime) stage runs elsewhere.
double fft_ring_cost(const RingDesc& r, bool pre) {
    double per_layer = 4.0 * r.n;
    for (int s2 = (pre && r.pre) ? 1 : 0; s2 < r.nfac; ++s2)
        per_layer += r.fac[s2] > 8 ? 2.0 * r.n * ((r.fac[s2] - 1) / 2 + kPrimeGroup - 1) / kPrimeGroup * kPrimeGroup
                                   : 3.0 * r.n;
    return per_layer;
}

// FFT work list: one CTA per (ring, chunk of layers), issued costliest first so that the
// last wave holds the cheapest CTAs.
std::vector<int2> fft_item_order(const Plan& p, bool pre) {
    std::vector<std::pair<double, int2>> fitems;
    const int kmax = std::max(1, p.d.nlayers);
    for (int j = 0; j < (int)p.h_rings.size(); ++j) {
        const RingDesc& r = p.h_rings[j];
        const double per_layer = fft_ring_cost(r, pre);
        for (int ci = 0; ci * r.chunk < kmax; ++ci) {
            const int c = std::min(r.chunk, kmax - ci * r.chunk);
            fitems.push_back({c * per_layer, make_int2(j, ci)});
        }
    }
    std::stable_sort(fitems.begin(), fitems.end(),
                     [](const std::pair<double, int2>& a, const std::pair<double, int2>& b) { return a.first > b.first; });
    std::vector<int2> out;
    for (auto& f : fitems) out.push_back(f.second);
    return out;
}

// Turns the tensor-core first stages on or off and reorders the FFT work list for it.
cudaError_t apply_prime_mode(Plan& p, int mode) {
    cudaError_t e = prime_set_mode(p, mode);
    if (e != cudaSuccess) return e;
    const std::vector<int2> items = fft_item_order(p, p.prime_mode != 0);
    return cudaMemcpy(p.d_fft_items, items.data(), items.size() * sizeof(int2), cudaMemcpyHostToDevice);
}

// Table block of a prime stage p > 8 (layout and use in sht_fft.cu, stage_prime):
// T[e] = (cos, sin)(2 pi g^(e - hpad + 1) / p) for e < 2 hpad, q_b = g^-b, r_a = g^a.
static int primitive_root(int p) {
    std::vector<int> qs;
    int m = p - 1;
    for (int d = 2; d * d <= m; ++d)
        if (m % d == 0) {
            qs.push_back(d);
            while (m % d == 0) m /= d;
        }
    if (m > 1) qs.push_back(m);
    auto pw = [p](int64_t b, int64_t e) {
        int64_t r = 1;
        b %= p;
        for (; e > 0; e >>= 1, b = b * b % p)
            if (e & 1) r = r * b % p;
        return r;
    };
    for (int g = 2; g < p; ++g) {
        bool ok = true;
        for (int q : qs) ok = ok && pw(g, (p - 1) / q) != 1;
        if (ok) return g;
    }
    return 1;
}

static void prime_table(int p, std::vector<float2>& out) {
    const int h = (p - 1) / 2, hpad = (h + kPrimeGroup - 1) / kPrimeGroup * kPrimeGroup;
    const int g = primitive_root(p);
    std::vector<int64_t> gp(p - 1);           // g^t mod p, t < p - 1
    gp[0] = 1;
    for (int t = 1; t < p - 1; ++t) gp[t] = gp[t - 1] * g % p;
    auto gpow = [&](int64_t t) { return gp[((t % (p - 1)) + (p - 1)) % (p - 1)]; };
    for (int e = 0; e < 2 * hpad; ++e) {
        const double a = 2.0 * M_PI * (double)gpow(e - hpad + 1) / p;
        out.push_back(make_float2((float)std::cos(a), (float)std::sin(a)));
    }
    std::vector<int32_t> idx(2 * hpad, 0);    // q_b | r_a
    for (int b = 0; b < h; ++b) idx[b] = (int32_t)gpow(-b);
    for (int a = 0; a < h; ++a) idx[hpad + a] = (int32_t)gpow(a);
    for (int e = 0; e < hpad; ++e) {
        float2 v;
        std::memcpy(&v.x, &idx[2 * e], 4);
        std::memcpy(&v.y, &idx[2 * e + 1], 4);
        out.push_back(v);
    }
}

int shortcut_mt(int kind, int nlon, double latd) {
    switch (kind) {
        case SHT_SHORTCUT_LINEAR: return nlon / 2;
        case SHT_SHORTCUT_QUADRATIC: return nlon / 3;
        case SHT_SHORTCUT_CUBIC: return nlon / 4;
        case SHT_SHORTCUT_LINQUADCOSLAT2: {
            const double c = std::cos(latd * M_PI / 180.0);
            return (int)std::floor(nlon / (2.0 + c * c));
        }
        case SHT_SHORTCUT_LINCUBCOSLAT: {
            const double c = std::cos(latd * M_PI / 180.0);
            return (int)std::floor(nlon / (2.0 + 2.0 * c));
        }
        default: return -1;
    }
}

template <class T>
cudaError_t upload(T** dst, const std::vector<T>& src, int64_t& bytes) {
    const size_t nb = std::max<size_t>(1, src.size()) * sizeof(T);
    cudaError_t e = cudaMalloc((void**)dst, nb);
    if (e != cudaSuccess) return e;
    bytes += (int64_t)nb;
    if (!src.empty()) e = cudaMemcpy(*dst, src.data(), src.size() * sizeof(T), cudaMemcpyHostToDevice);
    return e;
}

void release(Plan& p) {
    tc_release(p);
    prime_release(p);
    void* ptrs[] = {p.d_rings, p.d_twiddle, p.d_lam, p.d_lam_off, p.d_j0, p.d_rows, p.d_lm_off, p.d_syn_items,
                    p.d_ana_items, p.d_mt, p.d_gofs, p.d_grad, p.d_l_of, p.d_m_of, p.d_eig, p.d_eig_inv, p.d_four,
                    p.d_err, p.d_fft_items};
    for (void* q : ptrs)
        if (q) cudaFree(q);
}

struct DeviceGuard {
    int prev = -1;
    bool ok = true;
    explicit DeviceGuard(int dev) {
        if (cudaGetDevice(&prev) != cudaSuccess) {
            ok = false;
            return;
        }
        if (prev != dev && cudaSetDevice(dev) != cudaSuccess) ok = false;
    }
    ~DeviceGuard() {
        int cur = -1;
        if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
    }
};

int build_plan(Plan& p) {
    const sht_desc& d = p.d;
    p.nh = d.nlat_half;
    p.nlat = 2 * d.nlat_half;
    p.lmax = d.lmax;
    p.mmax = d.mmax;
    const int nh = p.nh;
    p.nlm = (int64_t)p.lmax * p.mmax - (int64_t)p.mmax * (p.mmax - 1) / 2;

    // --- grid (RingGrids) ---
    std::vector<int32_t> half(nh);
    for (int j = 0; j < nh; ++j)
        half[j] = d.grid == SHT_GRID_FULL_GAUSSIAN ? 4 * nh : 16 + 4 * (j + 1);  // full_gaussian.jl:45,
                                                                                // octahedral_gaussian.jl:64-70
    p.nlons.resize(p.nlat);
    for (int j = 0; j < nh; ++j) {
        p.nlons[j] = half[j];
        p.nlons[p.nlat - 1 - j] = half[j];
    }
    std::vector<int64_t> ring_start(p.nlat + 1, 0);
    for (int j = 0; j < p.nlat; ++j) ring_start[j + 1] = ring_start[j] + p.nlons[j];
    p.npoints = ring_start[p.nlat];
    p.nlon_max = *std::max_element(p.nlons.begin(), p.nlons.end());
    p.nfreq_max = p.nlon_max / 2 + 1;

    std::vector<double> x, w;
    gauss_legendre(p.nlat, x, w);
    p.latd.resize(p.nlat);
    p.weights = w;
    for (int j = 0; j < p.nlat; ++j) p.latd[j] = std::acos(x[j]) * 180.0 / M_PI - 90.0;  // full_gaussian.jl:48-50

    // --- Legendre shortcut (spectral_transform.jl:154-155) ---
    p.mt.resize(nh);
    for (int j = 0; j < nh; ++j) {
        const int t = shortcut_mt(d.shortcut, half[j], p.latd[j]);
        if (t < 0) return fail(SHT_EINVAL, "unknown Legendre shortcut %d", d.shortcut);
        p.mt[j] = std::min(t, p.mmax - 1);
    }
    p.j0.assign(p.mmax, nh);
    for (int m = 0; m < p.mmax; ++m)
        for (int j = 0; j < nh; ++j)
            if (p.mt[j] >= m) {
                p.j0[m] = j;
                break;
            }

    // --- spectral layout + Legendre table layout ---
    p.lm_off.resize(p.mmax);
    p.rows.resize(p.mmax);
    p.lam_off.resize(p.mmax);
    p.nh_pad = (nh + 63) / 64 * 64;
    int64_t lo = 0;
    for (int m = 0; m < p.mmax; ++m) {
        p.lm_off[m] = (int64_t)m * p.lmax - (int64_t)m * (m - 1) / 2;
        p.rows[m] = (p.lmax - m + 1) / 2;
        p.lam_off[m] = lo;
        lo += 2LL * p.rows[m] * p.nh_pad;
    }
    const int64_t lam_elems = lo;

    // --- Legendre polynomials in FP64, stored FP32: [m][parity][row][nh_pad] ---
    // lambda_lm (4pi-orthonormal, Condon-Shortley phase), the arithmetic of
    // AssociatedLegendrePolynomials.lambdalm! called at spectral_transform.jl:167-172.
    std::vector<float> lam((size_t)lam_elems, 0.0f);
    {
        const int nthreads = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
        auto work = [&](int tid) {
            std::vector<double> col(p.lmax);
            for (int j = tid; j < nh; j += nthreads) {
                const double colat = M_PI / 2 - p.latd[j] * M_PI / 180.0;   // grid.jl:142-143
                const double xc = std::cos(colat);
                const double s = std::sqrt(std::max(0.0, 1.0 - xc * xc));
                double pmm = 1.0 / std::sqrt(4.0 * M_PI);
                for (int m = 0; m <= p.mt[j]; ++m) {
                    if (m > 0) pmm = -std::sqrt((2.0 * m + 1.0) / (2.0 * m)) * s * pmm;
                    const int L = p.lmax - m;
                    col[0] = pmm;
                    if (L >= 2) {
                        double p0 = pmm, p1 = std::sqrt(2.0 * m + 3.0) * xc * pmm;
                        col[1] = p1;
                        double a_prev = std::sqrt((4.0 * (m + 1) * (m + 1) - 1.0) / ((m + 1.0) * (m + 1.0) - 1.0 * m * m));
                        for (int l = m + 2; l < p.lmax; ++l) {
                            const double a = std::sqrt((4.0 * l * l - 1.0) / (1.0 * l * l - 1.0 * m * m));
                            const double p2 = a * (xc * p1 - p0 / a_prev);
                            col[l - m] = p2;
                            p0 = p1;
                            p1 = p2;
                            a_prev = a;
                        }
                    }
                    float* base = lam.data() + p.lam_off[m];
                    for (int i = 0; i < L; ++i) {
                        const int par = i & 1, row = i >> 1;
                        base[((int64_t)par * p.rows[m] + row) * p.nh_pad + j] = (float)col[i];
                    }
                }
            }
        };
        std::vector<std::thread> th;
        for (int t = 0; t < nthreads; ++t) th.emplace_back(work, t);
        for (auto& t : th) t.join();
    }

    // --- per-ring FFT descriptors and twiddles (FP64 -> FP32) ---
    std::vector<RingDesc> rings(nh);
    std::vector<float2> tw;
    int64_t gofs = 0;
    const int smem_budget = kFftSmemBudget;
    int max_smem = 0;
    p.min_chunk = 1 << 30;
    for (int j = 0; j < nh; ++j) {
        RingDesc& r = rings[j];
        std::memset(&r, 0, sizeof r);
        r.n = half[j];
        r.mt = p.mt[j];
        r.nfac = factorize(r.n, r.fac);
        if (r.nfac < 0) return fail(SHT_EINVAL, "ring length %d has too many factors", r.n);
        r.off_north = ring_start[j];
        r.off_south = ring_start[p.nlat - 1 - j];
        r.gofs = gofs;
        gofs += r.mt + 1;
        r.tw_off = (int64_t)tw.size();
        for (int t = 0; t < r.n; ++t) {
            const double a = -2.0 * M_PI * t / r.n;
            tw.push_back(make_float2((float)std::cos(a), (float)std::sin(a)));
        }
        if (r.n % 2) tw.push_back(make_float2(0.f, 0.f));
        for (int s = 0; s < r.nfac; ++s)
            if (r.fac[s] > 8) prime_table(r.fac[s], tw);
        r.gen_len = (int32_t)((int64_t)tw.size() - r.tw_off - ((r.n + 1) & ~1));
        r.domega = (float)(p.weights[j] * (2.0 * M_PI / r.n));                  // quadrature_weights.jl:48-49
        r.coslat_inv = (float)(1.0 / std::cos(p.latd[j] * M_PI / 180.0));       // spectral_transform.jl:150-151
        p.coslat_inv_max = std::max(p.coslat_inv_max, r.coslat_inv);
        // shared memory of the FFT kernels: twiddles, prime tables and two buffers of
        // chunk x n complex
        const int tw_bytes = (((r.n + 1) & ~1) + r.gen_len) * 8;
        // layer stride ldx = n + pad with ldx = 16 / chunk (mod 16) in float2 units (2 for
        // chunks of 8 or more): the chunk's layers of one order then fall in distinct
        // shared-memory banks when the lanes run over the layers
        // (and ldx >= 2 (mt + 1): the synthesis stages the ring's scratch rows in one buffer)
        auto stride = [&](int c) {
            const int want = c >= 8 ? 2 : 16 / c;
            const int base = std::max(r.n, 2 * (r.mt + 1));
            return base + (((want - base) % 16) + 16) % 16;
        };
        int chunk = 1;
        while (chunk * 2 <= 32 && tw_bytes + 2 * (chunk * 2) * stride(chunk * 2) * 8 <= smem_budget) chunk *= 2;
        r.chunk = chunk;
        r.ldx = stride(chunk);
        p.min_chunk = std::min(p.min_chunk, chunk);
        max_smem = std::max(max_smem, tw_bytes + 2 * chunk * r.ldx * 8);
    }
    p.scratch_rows = gofs;
    p.smem_fft = max_smem;

    // rings whose first stage may run on the tensor cores (sht_prime_tc.cu)
    const int64_t ymid_elems = prime_mark_rings(rings, d.nlayers);
    p.h_rings = rings;
    p.h_ring_cost.assign(nh, 0.0);
    for (int j = 0; j < nh; ++j) p.h_ring_cost[j] = fft_ring_cost(rings[j], false);
    const std::vector<int2> fft_items = fft_item_order(p, false);

    // --- work lists of the Legendre kernels (64-row tiles, heavy orders first) ---
    std::vector<LegItem> syn, ana;
    for (int m = 0; m < p.mmax; ++m) {
        if (p.j0[m] < nh)
            for (int t = p.j0[m] / 64; t * 64 < nh; ++t) syn.push_back({m, t});
        for (int t = 0; t * 64 < p.rows[m]; ++t) ana.push_back({m, t});   // every coefficient is written
    }

    // --- spectral operator factors (gradient_arrays.jl:1-215) in FP64 -> FP32 ---
    const int64_t nlm = p.nlm;
    std::vector<float> grad((size_t)G_COUNT * nlm, 0.0f);
    std::vector<int32_t> l_of(nlm), m_of(nlm);
    auto eps = [](double l, double m) { return std::sqrt((l * l - m * m) / (4.0 * l * l - 1.0)); };
    for (int m = 0; m < p.mmax; ++m)
        for (int l = m; l < p.lmax; ++l) {
            const int64_t lm = p.lm_off[m] + (l - m);
            l_of[lm] = l;
            m_of[lm] = m;
            const bool last = (l == p.lmax - 1);
            const double L1 = l + 1.0;                 // 1-based degree
            const double e_l = (l == 0 && m == 0) ? 0.0 : eps(l, m);
            const double e_lp = eps(l + 1.0, m);
            grad[G_GRAD_Y1 * nlm + lm] = (float)(-(L1 - 2.0) * e_l);
            grad[G_GRAD_Y2 * nlm + lm] = last ? 0.f : (float)((L1 + 1.0) * e_lp);
            grad[G_GRAD_Y_VORDIV1 * nlm + lm] = last ? 0.f : (float)(L1 * e_l);
            grad[G_GRAD_Y_VORDIV2 * nlm + lm] = last ? 0.f : (float)((L1 - 1.0) * e_lp);
            grad[G_GRAD_X_VORDIV * nlm + lm] = last ? 0.f : (float)m;
            grad[G_VORDIV_TO_UV_X * nlm + lm] = (lm == 0) ? 0.f : (float)(-m / (L1 * (L1 - 1.0)));
            grad[G_VORDIV_TO_UV1 * nlm + lm] = (lm == 0) ? 0.f : (float)(e_l / (L1 - 1.0));
            grad[G_VORDIV_TO_UV2 * nlm + lm] = last ? 0.f : (float)(e_lp / L1);
        }
    std::vector<float> eig(p.lmax), eig_inv(p.lmax);
    for (int l = 0; l < p.lmax; ++l) {
        const double e = -(double)l * (l + 1.0);
        eig[l] = (float)e;
        eig_inv[l] = l == 0 ? 0.f : (float)(1.0 / e);     // gradient_arrays.jl:165-170
    }

    // --- device upload ---
    int64_t tb = 0;
    cudaError_t e;
#define UP(dst, src)                                          \
    if ((e = upload(&(dst), (src), tb)) != cudaSuccess) {     \
        return cuda_fail(e, "sht_plan_create upload " #dst); \
    }
    UP(p.d_rings, rings);
    UP(p.d_twiddle, tw);
    UP(p.d_lam, lam);
    UP(p.d_lam_off, p.lam_off);
    UP(p.d_j0, p.j0);
    UP(p.d_rows, p.rows);
    UP(p.d_lm_off, p.lm_off);
    UP(p.d_syn_items, syn);
    UP(p.d_ana_items, ana);
    UP(p.d_fft_items, fft_items);
    UP(p.d_mt, p.mt);
    UP(p.d_grad, grad);
    UP(p.d_l_of, l_of);
    UP(p.d_m_of, m_of);
    UP(p.d_eig, eig);
    UP(p.d_eig_inv, eig_inv);
#undef UP
    std::vector<int64_t> gofs_v(nh);
    for (int j = 0; j < nh; ++j) gofs_v[j] = rings[j].gofs;
    if ((e = upload(&p.d_gofs, gofs_v, tb)) != cudaSuccess) return cuda_fail(e, "sht_plan_create upload gofs");
    p.n_syn_items = (int)syn.size();
    p.n_ana_items = (int)ana.size();
    p.n_fft_items = (int)fft_items.size();
    p.h_syn_items = syn;
    p.h_ana_items = ana;
    p.table_bytes = tb;

    p.four_elems = p.scratch_rows * 2 * std::max(1, d.nlayers);
    if ((e = cudaMalloc((void**)&p.d_four, p.four_elems * sizeof(float2))) != cudaSuccess)
        return cuda_fail(e, "sht_plan_create scratch");
    if ((e = cudaMalloc((void**)&p.d_err, sizeof(int32_t))) != cudaSuccess) return cuda_fail(e, "sht_plan_create");
    if ((e = cudaMemset(p.d_err, 0, sizeof(int32_t))) != cudaSuccess) return cuda_fail(e, "sht_plan_create");
    if ((e = fft_set_smem(p.smem_fft)) != cudaSuccess) return cuda_fail(e, "sht_plan_create fft smem");
    if (d.precision != SHT_PREC_FP32) {
        if (!tc_supported()) return fail(SHT_EUNSUPPORTED, "tensor-core Legendre precision %d not available", d.precision);
        if ((e = tc_prepare(p)) != cudaSuccess) return cuda_fail(e, "sht_plan_create tensor-core tables");
    }
    if ((e = fused_prepare(p)) != cudaSuccess) return cuda_fail(e, "sht_plan_create fused kernels");
    // the tensor-core prime stages (off until sht_plan_set_prime_stage turns them on)
    if ((e = prime_create(p, ymid_elems)) != cudaSuccess) return cuda_fail(e, "sht_plan_create prime stages");
    return SHT_OK;
}

bool ok_ptr(const void* q) { return q != nullptr; }

int check_call(const sht_plan* plan, int K, const char* what) {
    if (!plan) return fail(SHT_EINVAL, "%s: plan is NULL", what);
    if (K < 0 || K > plan->p.d.nlayers)
        return fail(SHT_EINVAL, "%s: DimensionMismatch: K = %d layers, plan has nlayers = %d", what, K,
                    plan->p.d.nlayers);
    return SHT_OK;
}

int check_ldc(const Plan& p, int64_t ldc, const char* what) {
    if (ldc < p.nlm)
        return fail(SHT_EINVAL, "%s: DimensionMismatch: leading dimension %lld < nlm = %lld (lmax=%d, mmax=%d)", what,
                    (long long)ldc, (long long)p.nlm, p.lmax, p.mmax);
    return SHT_OK;
}

int check_ldg(const Plan& p, int64_t ldg, const char* what) {
    if (ldg < p.npoints)
        return fail(SHT_EINVAL, "%s: DimensionMismatch: leading dimension %lld < npoints = %lld", what, (long long)ldg,
                    (long long)p.npoints);
    return SHT_OK;
}

int finish(cudaError_t e, const char* what) {
    if (e != cudaSuccess) return cuda_fail(e, what);
    return SHT_OK;
}

cudaError_t legendre_synthesis(const Plan& p, const float2* coeffs, int64_t ldc, int K, cudaStream_t s) {
    if (p.d.precision == SHT_PREC_FP32) return launch_legendre_synthesis_fp32(p, coeffs, ldc, K, s);
    return launch_legendre_synthesis_tc(p, coeffs, ldc, K, s);
}

cudaError_t legendre_analysis(const Plan& p, float2* coeffs, int64_t ldc, int K, bool add, cudaStream_t s) {
    if (p.d.precision == SHT_PREC_FP32) return launch_legendre_analysis_fp32(p, coeffs, ldc, K, add, s);
    return launch_legendre_analysis_tc(p, coeffs, ldc, K, add, s);
}

}  // namespace

extern "C" {

const char* sht_last_error(void) { return g_last_error.c_str(); }
const char* sht_version(void) { return "libsht 0.1 (sm_100a)"; }

int sht_plan_create(const sht_desc* desc, sht_plan** out) {
    if (!desc || !out) return fail(SHT_EINVAL, "sht_plan_create: NULL argument");
    *out = nullptr;
    const sht_desc& d = *desc;
    if (d.grid != SHT_GRID_FULL_GAUSSIAN && d.grid != SHT_GRID_OCTAHEDRAL_GAUSSIAN)
        return fail(SHT_EUNSUPPORTED, "grid kind %d not supported (full or octahedral Gaussian only)", d.grid);
    if (d.nlat_half < 1 || d.nlat_half > 8192) return fail(SHT_EINVAL, "nlat_half %d out of range", d.nlat_half);
    if (d.mmax < 1 || d.lmax < d.mmax || d.lmax > 8192)
        return fail(SHT_EINVAL, "spectrum lmax=%d mmax=%d invalid (need 1 <= mmax <= lmax)", d.lmax, d.mmax);
    if (d.nlayers < 1) return fail(SHT_EINVAL, "nlayers %d must be >= 1", d.nlayers);
    if (d.precision < SHT_PREC_FP32 || d.precision > SHT_PREC_BF16X5)
        return fail(SHT_EINVAL, "precision %d unknown", d.precision);
    if (d.precision != SHT_PREC_FP32 && d.nlayers > 1024)
        return fail(SHT_EINVAL, "tensor-core precisions support nlayers <= 1024");
    DeviceGuard g(d.device);
    if (!g.ok) return fail(SHT_ECUDA, "sht_plan_create: cannot select device %d", d.device);
    sht_plan* h = new (std::nothrow) sht_plan();
    if (!h) return fail(SHT_ENOMEM, "sht_plan_create: host allocation failed");
    h->p.d = d;
    h->p.device = d.device;
    const int rc = build_plan(h->p);
    if (rc != SHT_OK) {
        release(h->p);
        delete h;
        return rc;
    }
    *out = h;
    return SHT_OK;
}

static void release_host(HostPipe& h) {
    if (h.copy_in) cudaStreamSynchronize(h.copy_in);
    if (h.copy_out) cudaStreamSynchronize(h.copy_out);
    for (int i = 0; i < 2; ++i) {
        if (h.in_slot[i]) cudaFree(h.in_slot[i]);
        if (h.out_slot[i]) cudaFree(h.out_slot[i]);
        cudaEvent_t* ev[] = {&h.in_ready[i], &h.in_free[i], &h.out_ready[i], &h.out_free[i]};
        for (cudaEvent_t* e : ev)
            if (*e) cudaEventDestroy(*e);
    }
    if (h.copy_in) cudaStreamDestroy(h.copy_in);
    if (h.copy_out) cudaStreamDestroy(h.copy_out);
    h = HostPipe{};
}

int sht_plan_destroy(sht_plan* plan) {
    if (!plan) return SHT_OK;
    DeviceGuard g(plan->p.device);
    release_host(plan->host);
    release(plan->p);
    delete plan;
    return SHT_OK;
}

int sht_plan_info(const sht_plan* plan, sht_info* info) {
    if (!plan || !info) return fail(SHT_EINVAL, "sht_plan_info: NULL argument");
    const Plan& p = plan->p;
    info->npoints = p.npoints;
    info->nlm = p.nlm;
    info->nlat = p.nlat;
    info->nlat_half = p.nh;
    info->nlon_max = p.nlon_max;
    info->nfreq_max = p.nfreq_max;
    info->lmax = p.lmax;
    info->mmax = p.mmax;
    info->nlayers = p.d.nlayers;
    info->precision = p.d.precision;
    info->scratch_bytes = p.four_elems * (int64_t)sizeof(float2);
    info->table_bytes = p.table_bytes;
    return SHT_OK;
}

int sht_plan_tables(const sht_plan* plan, double* latd, double* weights, int32_t* nlons, int32_t* mmax_truncation) {
    if (!plan) return fail(SHT_EINVAL, "sht_plan_tables: NULL plan");
    const Plan& p = plan->p;
    if (latd) std::memcpy(latd, p.latd.data(), p.nlat * sizeof(double));
    if (weights) std::memcpy(weights, p.weights.data(), p.nlat * sizeof(double));
    if (nlons) std::memcpy(nlons, p.nlons.data(), p.nlat * sizeof(int32_t));
    if (mmax_truncation) std::memcpy(mmax_truncation, p.mt.data(), p.nh * sizeof(int32_t));
    return SHT_OK;
}

int sht_plan_autotune(sht_plan* plan, int K, void* stream, int32_t* tile_columns) {
    int rc;
    if ((rc = check_call(plan, K, "sht_plan_autotune")) != SHT_OK) return rc;
    if (tile_columns) tile_columns[0] = tile_columns[1] = 0;
    Plan& p = plan->p;
    if (K == 0) return SHT_OK;
    DeviceGuard g(p.device);
    cudaStream_t s = (cudaStream_t)stream;
    const bool tc = p.d.precision != SHT_PREC_FP32;
    float2* c = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaError_t e = cudaMalloc(&c, p.nlm * K * sizeof(float2));
    if (e == cudaSuccess) e = cudaMemsetAsync(c, 0, p.nlm * K * sizeof(float2), s);
    if (e == cudaSuccess) e = cudaEventCreate(&e0);
    if (e == cudaSuccess) e = cudaEventCreate(&e1);
    auto time = [&](auto&& launch, float& ms) {
        for (int w = 0; w < 2 && e == cudaSuccess; ++w) e = launch();
        if (e == cudaSuccess) e = cudaEventRecord(e0, s);
        for (int r = 0; r < 5 && e == cudaSuccess; ++r) e = launch();
        if (e == cudaSuccess) e = cudaEventRecord(e1, s);
        if (e == cudaSuccess) e = cudaEventSynchronize(e1);
        if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
    };
    int best[2] = {p.leg_bn_syn, p.leg_bn_ana};
    if (tc) {
        // tcgen05 column tile width: one width serves both directions (the images are laid out for it)
        best[0] = best[1] = tc_tile_cols(p);
        float best_ms = 1e30f;
        for (int cols : {128, 64}) {
            if (cols == 64 && 2 * K <= 64) break;       // a single tile of <= 64 columns either way
            tc_set_tile_cols(p, cols);
            float ms = 0.f;
            time([&]() {
                cudaError_t x = legendre_synthesis(p, c, p.nlm, K, s);
                return x == cudaSuccess ? legendre_analysis(p, c, p.nlm, K, false, s) : x;
            }, ms);
            if (e == cudaSuccess && ms < best_ms) {
                best_ms = ms;
                best[0] = best[1] = cols;
            }
        }
        tc_set_tile_cols(p, best[0]);
    } else {
        for (int dir = 0; dir < 2 && e == cudaSuccess; ++dir) {
            float best_ms = 1e30f;
            for (int bn : {32, 64, 128}) {
                (dir == 0 ? p.leg_bn_syn : p.leg_bn_ana) = bn;
                float ms = 0.f;
                time([&]() {
                    return dir == 0 ? launch_legendre_synthesis_fp32(p, c, p.nlm, K, s)
                                    : launch_legendre_analysis_fp32(p, c, p.nlm, K, false, s);
                }, ms);
                if (e == cudaSuccess && ms < best_ms) {
                    best_ms = ms;
                    best[dir] = bn;
                }
            }
        }
        p.leg_bn_syn = best[0];
        p.leg_bn_ana = best[1];
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (c) cudaFree(c);
    if (e != cudaSuccess) return cuda_fail(e, "sht_plan_autotune");
    if (tile_columns) {
        tile_columns[0] = best[0];
        tile_columns[1] = best[1];
    }
    return SHT_OK;
}

int sht_plan_set_tile_columns(sht_plan* plan, int synthesis, int analysis) {
    if (!plan) return fail(SHT_EINVAL, "sht_plan_set_tile_columns: NULL plan");
    Plan& p = plan->p;
    if (p.d.precision == SHT_PREC_FP32) {
        auto ok = [](int v) { return v == 32 || v == 64 || v == 128; };
        if (!ok(synthesis) || !ok(analysis))
            return fail(SHT_EINVAL, "sht_plan_set_tile_columns: FP32 plans take 32, 64 or 128 columns");
        p.leg_bn_syn = synthesis;
        p.leg_bn_ana = analysis;
        return SHT_OK;
    }
    if (synthesis != analysis || !tc_set_tile_cols(p, synthesis))
        return fail(SHT_EINVAL, "sht_plan_set_tile_columns: tensor-core plans take 64 or 128 columns, the same for "
                                "both directions");
    return SHT_OK;
}

int sht_plan_set_prime_stage(sht_plan* plan, int mode) {
    if (!plan) return fail(SHT_EINVAL, "sht_plan_set_prime_stage: NULL plan");
    if (mode != SHT_PRIME_DIRECT && mode != SHT_PRIME_TENSOR)
        return fail(SHT_EINVAL, "sht_plan_set_prime_stage: mode %d is neither SHT_PRIME_DIRECT nor SHT_PRIME_TENSOR",
                    mode);
    if (mode == SHT_PRIME_TENSOR && !tc_supported())
        return fail(SHT_EUNSUPPORTED, "sht_plan_set_prime_stage: tensor cores (sm_100) not available");
    DeviceGuard g(plan->p.device);
    const cudaError_t e = apply_prime_mode(plan->p, mode);
    return e == cudaSuccess ? SHT_OK : cuda_fail(e, "sht_plan_set_prime_stage");
}

int sht_plan_get_prime_stage(const sht_plan* plan, int32_t* mode, int32_t* available) {
    if (!plan) return fail(SHT_EINVAL, "sht_plan_get_prime_stage: NULL plan");
    if (mode) *mode = plan->p.prime_mode;
    if (available) *available = prime_available(plan->p) ? 1 : 0;
    return SHT_OK;
}

int sht_plan_set_fusion(sht_plan* plan, int mode) {
    if (!plan) return fail(SHT_EINVAL, "sht_plan_set_fusion: NULL plan");
    if (mode != SHT_FUSION_OFF && mode != SHT_FUSION_ON)
        return fail(SHT_EINVAL, "sht_plan_set_fusion: mode %d is neither SHT_FUSION_OFF nor SHT_FUSION_ON", mode);
    Plan& p = plan->p;
    if (mode == SHT_FUSION_ON && !p.fusion_ok)
        return fail(SHT_EUNSUPPORTED, "sht_plan_set_fusion: %s", p.tc ? "tensor-core plans keep the separate kernels"
                                                                    : "the plan's cluster data exceeds shared memory");
    p.fusion = mode;
    return SHT_OK;
}

int sht_plan_get_fusion(const sht_plan* plan, int32_t* mode, int32_t* available) {
    if (!plan) return fail(SHT_EINVAL, "sht_plan_get_fusion: NULL plan");
    if (mode) *mode = plan->p.fusion;
    if (available) *available = plan->p.fusion_ok;
    return SHT_OK;
}

int sht_device_status(sht_plan* plan, int32_t* status) {
    if (!plan || !status) return fail(SHT_EINVAL, "sht_device_status: NULL argument");
    DeviceGuard g(plan->p.device);
    cudaError_t e = cudaDeviceSynchronize();
    if (e != cudaSuccess) return cuda_fail(e, "sht_device_status");
    if ((e = cudaMemcpy(status, plan->p.d_err, sizeof(int32_t), cudaMemcpyDeviceToHost)) != cudaSuccess)
        return cuda_fail(e, "sht_device_status");
    if ((e = cudaMemset(plan->p.d_err, 0, sizeof(int32_t))) != cudaSuccess) return cuda_fail(e, "sht_device_status");
    return SHT_OK;
}

int sht_diag_wait_expiry(sht_plan* plan, int32_t limit_us, void* stream) {
    if (!plan) return fail(SHT_EINVAL, "sht_diag_wait_expiry: NULL plan");
    if (limit_us < 1 || limit_us > 1000000)
        return fail(SHT_EINVAL, "sht_diag_wait_expiry: limit_us = %d outside 1 .. 1000000", (int)limit_us);
    DeviceGuard g(plan->p.device);
    const cudaError_t e = launch_wait_probe(plan->p.d_err, (uint64_t)limit_us * 1000u, (cudaStream_t)stream);
    return e == cudaSuccess ? SHT_OK : cuda_fail(e, "sht_diag_wait_expiry");
}

int sht_legendre_synthesis(sht_plan* plan, const void* coeffs, int64_t ldc, int K, void* stream) {
    int rc;
    if ((rc = check_call(plan, K, "sht_legendre_synthesis")) != SHT_OK) return rc;
    if ((rc = check_ldc(plan->p, ldc, "sht_legendre_synthesis")) != SHT_OK) return rc;
    if (K == 0) return SHT_OK;
    if (!ok_ptr(coeffs)) return fail(SHT_EINVAL, "sht_legendre_synthesis: NULL coeffs");
    DeviceGuard g(plan->p.device);
    return finish(legendre_synthesis(plan->p, (const float2*)coeffs, ldc, K, (cudaStream_t)stream),
                  "sht_legendre_synthesis");
}

int sht_fourier_synthesis(sht_plan* plan, float* grid, int64_t ldg, int K, unsigned flags, void* stream) {
    int rc;
    if ((rc = check_call(plan, K, "sht_fourier_synthesis")) != SHT_OK) return rc;
    if ((rc = check_ldg(plan->p, ldg, "sht_fourier_synthesis")) != SHT_OK) return rc;
    if (K == 0) return SHT_OK;
    if (!ok_ptr(grid)) return fail(SHT_EINVAL, "sht_fourier_synthesis: NULL grid");
    DeviceGuard g(plan->p.device);
    return finish(launch_fft_synthesis(plan->p, grid, ldg, K, flags, (cudaStream_t)stream), "sht_fourier_synthesis");
}

int sht_fourier_analysis(sht_plan* plan, const float* grid, int64_t ldg, int K, void* stream) {
    int rc;
    if ((rc = check_call(plan, K, "sht_fourier_analysis")) != SHT_OK) return rc;
    if ((rc = check_ldg(plan->p, ldg, "sht_fourier_analysis")) != SHT_OK) return rc;
    if (K == 0) return SHT_OK;
    if (!ok_ptr(grid)) return fail(SHT_EINVAL, "sht_fourier_analysis: NULL grid");
    DeviceGuard g(plan->p.device);
    return finish(launch_fft_analysis(plan->p, grid, ldg, K, (cudaStream_t)stream), "sht_fourier_analysis");
}

int sht_legendre_analysis(sht_plan* plan, void* coeffs, int64_t ldc, int K, unsigned flags, void* stream) {
    int rc;
    if ((rc = check_call(plan, K, "sht_legendre_analysis")) != SHT_OK) return rc;
    if ((rc = check_ldc(plan->p, ldc, "sht_legendre_analysis")) != SHT_OK) return rc;
    if (K == 0) return SHT_OK;
    if (!ok_ptr(coeffs)) return fail(SHT_EINVAL, "sht_legendre_analysis: NULL coeffs");
    DeviceGuard g(plan->p.device);
    return finish(legendre_analysis(plan->p, (float2*)coeffs, ldc, K, (flags & SHT_ADD) != 0, (cudaStream_t)stream),
                  "sht_legendre_analysis");
}

int sht_synthesize(sht_plan* plan, const void* coeffs, int64_t ldc, float* grid, int64_t ldg, int K, unsigned flags,
                   void* stream) {
    int rc;
    if ((rc = check_call(plan, K, "sht_synthesize")) != SHT_OK) return rc;
    if ((rc = check_ldc(plan->p, ldc, "sht_synthesize")) != SHT_OK) return rc;
    if ((rc = check_ldg(plan->p, ldg, "sht_synthesize")) != SHT_OK) return rc;
    if (K == 0) return SHT_OK;
    if (!ok_ptr(coeffs) || !ok_ptr(grid)) return fail(SHT_EINVAL, "sht_synthesize: NULL array");
    DeviceGuard g(plan->p.device);
    cudaStream_t s = (cudaStream_t)stream;
    if (plan->p.fusion)
        return finish(launch_fused_synthesis(plan->p, (const float2*)coeffs, ldc, grid, ldg, K, flags, s),
                      "sht_synthesize (fused)");
    cudaError_t e = legendre_synthesis(plan->p, (const float2*)coeffs, ldc, K, s);
    if (e != cudaSuccess) return cuda_fail(e, "sht_synthesize (Legendre)");
    return finish(launch_fft_synthesis(plan->p, grid, ldg, K, flags, s), "sht_synthesize (Fourier)");
}

int sht_analyze(sht_plan* plan, const float* grid, int64_t ldg, void* coeffs, int64_t ldc, int K, unsigned flags,
                void* stream) {
    int rc;
    if ((rc = check_call(plan, K, "sht_analyze")) != SHT_OK) return rc;
    if ((rc = check_ldc(plan->p, ldc, "sht_analyze")) != SHT_OK) return rc;
    if ((rc = check_ldg(plan->p, ldg, "sht_analyze")) != SHT_OK) return rc;
    if (K == 0) return SHT_OK;
    if (!ok_ptr(coeffs) || !ok_ptr(grid)) return fail(SHT_EINVAL, "sht_analyze: NULL array");
    DeviceGuard g(plan->p.device);
    cudaStream_t s = (cudaStream_t)stream;
    if (plan->p.fusion)
        return finish(launch_fused_analysis(plan->p, grid, ldg, (float2*)coeffs, ldc, K, (flags & SHT_ADD) != 0, s),
                      "sht_analyze (fused)");
    cudaError_t e = launch_fft_analysis(plan->p, grid, ldg, K, s);
    if (e != cudaSuccess) return cuda_fail(e, "sht_analyze (Fourier)");
    return finish(legendre_analysis(plan->p, (float2*)coeffs, ldc, K, (flags & SHT_ADD) != 0, s),
                  "sht_analyze (Legendre)");
}

// ---- host-buffer transforms -------------------------------------------------------
namespace {
constexpr int kDefaultHostChunk = 16;

cudaError_t host_prepare(sht_plan* plan, int chunk) {
    HostPipe& h = plan->host;
    chunk = std::max(1, std::min(chunk, std::max(1, plan->p.d.nlayers)));
    if (h.chunk == chunk) return cudaSuccess;
    release_host(h);
    h.chunk = chunk;
    const size_t bytes = (size_t)chunk * plan->p.nlm * sizeof(float2);
    cudaError_t e = cudaSuccess;
    for (int i = 0; i < 2 && e == cudaSuccess; ++i) {
        e = cudaMalloc((void**)&h.in_slot[i], bytes);
        if (e == cudaSuccess) e = cudaMalloc((void**)&h.out_slot[i], bytes);
        cudaEvent_t* ev[] = {&h.in_ready[i], &h.in_free[i], &h.out_ready[i], &h.out_free[i]};
        for (cudaEvent_t* q : ev)
            if (e == cudaSuccess) e = cudaEventCreateWithFlags(q, cudaEventDisableTiming);
    }
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&h.copy_in, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&h.copy_out, cudaStreamNonBlocking);
    if (e != cudaSuccess) release_host(h);
    return e;
}
}  // namespace

int sht_plan_set_host_chunk(sht_plan* plan, int layers) {
    if (!plan) return fail(SHT_EINVAL, "sht_plan_set_host_chunk: NULL plan");
    if (layers < 1) return fail(SHT_EINVAL, "sht_plan_set_host_chunk: layers must be >= 1");
    DeviceGuard g(plan->p.device);
    const cudaError_t e = host_prepare(plan, layers);
    return e == cudaSuccess ? SHT_OK : cuda_fail(e, "sht_plan_set_host_chunk");
}

int sht_synthesize_host(sht_plan* plan, const void* coeffs_host, int64_t ldc, float* grid, int64_t ldg, int K,
                        unsigned flags, void* stream) {
    int rc;
    if ((rc = check_call(plan, K, "sht_synthesize_host")) != SHT_OK) return rc;
    if ((rc = check_ldc(plan->p, ldc, "sht_synthesize_host")) != SHT_OK) return rc;
    if ((rc = check_ldg(plan->p, ldg, "sht_synthesize_host")) != SHT_OK) return rc;
    if (K == 0) return SHT_OK;
    if (!ok_ptr(coeffs_host) || !ok_ptr(grid)) return fail(SHT_EINVAL, "sht_synthesize_host: NULL array");
    DeviceGuard g(plan->p.device);
    cudaError_t e = plan->host.chunk ? cudaSuccess : host_prepare(plan, kDefaultHostChunk);
    if (e != cudaSuccess) return cuda_fail(e, "sht_synthesize_host (staging)");
    HostPipe& h = plan->host;
    const Plan& p = plan->p;
    cudaStream_t s = (cudaStream_t)stream;
    const float2* src = static_cast<const float2*>(coeffs_host);
    for (int k0 = 0; k0 < K && e == cudaSuccess; k0 += h.chunk) {
        const int c = std::min(h.chunk, K - k0);
        const int i = h.in_next;
        h.in_next ^= 1;
        // the slot's previous chunk has been read by its synthesis
        e = cudaStreamWaitEvent(h.copy_in, h.in_free[i], 0);
        if (e == cudaSuccess)
            e = cudaMemcpy2DAsync(h.in_slot[i], p.nlm * sizeof(float2), src + (int64_t)k0 * ldc, ldc * sizeof(float2),
                                  p.nlm * sizeof(float2), c, cudaMemcpyHostToDevice, h.copy_in);
        if (e == cudaSuccess) e = cudaEventRecord(h.in_ready[i], h.copy_in);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(s, h.in_ready[i], 0);
        if (e == cudaSuccess) e = legendre_synthesis(p, h.in_slot[i], p.nlm, c, s);
        if (e == cudaSuccess) e = launch_fft_synthesis(p, grid + (int64_t)k0 * ldg, ldg, c, flags, s);
        if (e == cudaSuccess) e = cudaEventRecord(h.in_free[i], s);
    }
    return finish(e, "sht_synthesize_host");
}

int sht_analyze_host(sht_plan* plan, const float* grid, int64_t ldg, void* coeffs_host, int64_t ldc, int K,
                     unsigned flags, void* stream) {
    int rc;
    if ((rc = check_call(plan, K, "sht_analyze_host")) != SHT_OK) return rc;
    if ((rc = check_ldc(plan->p, ldc, "sht_analyze_host")) != SHT_OK) return rc;
    if ((rc = check_ldg(plan->p, ldg, "sht_analyze_host")) != SHT_OK) return rc;
    if (flags & SHT_ADD) return fail(SHT_EINVAL, "sht_analyze_host: SHT_ADD into host memory is not supported");
    if (K == 0) return SHT_OK;
    if (!ok_ptr(coeffs_host) || !ok_ptr(grid)) return fail(SHT_EINVAL, "sht_analyze_host: NULL array");
    DeviceGuard g(plan->p.device);
    cudaError_t e = plan->host.chunk ? cudaSuccess : host_prepare(plan, kDefaultHostChunk);
    if (e != cudaSuccess) return cuda_fail(e, "sht_analyze_host (staging)");
    HostPipe& h = plan->host;
    const Plan& p = plan->p;
    cudaStream_t s = (cudaStream_t)stream;
    float2* dst = static_cast<float2*>(coeffs_host);
    for (int k0 = 0; k0 < K && e == cudaSuccess; k0 += h.chunk) {
        const int c = std::min(h.chunk, K - k0);
        const int i = h.out_next;
        h.out_next ^= 1;
        // the slot's previous chunk has reached the host
        e = cudaStreamWaitEvent(s, h.out_free[i], 0);
        if (e == cudaSuccess) e = launch_fft_analysis(p, grid + (int64_t)k0 * ldg, ldg, c, s);
        if (e == cudaSuccess) e = legendre_analysis(p, h.out_slot[i], p.nlm, c, false, s);
        if (e == cudaSuccess) e = cudaEventRecord(h.out_ready[i], s);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(h.copy_out, h.out_ready[i], 0);
        if (e == cudaSuccess)
            e = cudaMemcpy2DAsync(dst + (int64_t)k0 * ldc, ldc * sizeof(float2), h.out_slot[i], p.nlm * sizeof(float2),
                                  p.nlm * sizeof(float2), c, cudaMemcpyDeviceToHost, h.copy_out);
        if (e == cudaSuccess) e = cudaEventRecord(h.out_free[i], h.copy_out);
    }
    return finish(e, "sht_analyze_host");
}

int sht_host_wait(sht_plan* plan, void* stream) {
    if (!plan) return fail(SHT_EINVAL, "sht_host_wait: NULL plan");
    if (!plan->host.chunk) return SHT_OK;
    DeviceGuard g(plan->p.device);
    cudaError_t e = cudaSuccess;
    for (int i = 0; i < 2 && e == cudaSuccess; ++i) e = cudaStreamWaitEvent((cudaStream_t)stream, plan->host.out_free[i], 0);
    return finish(e, "sht_host_wait");
}

int sht_synthesize_adjoint(sht_plan* plan, const float* grid_bar, int64_t ldg, void* coeffs_bar, int64_t ldc, int K,
                           unsigned flags, void* stream) {
    int rc;
    if ((rc = check_call(plan, K, "sht_synthesize_adjoint")) != SHT_OK) return rc;
    if ((rc = check_ldc(plan->p, ldc, "sht_synthesize_adjoint")) != SHT_OK) return rc;
    if ((rc = check_ldg(plan->p, ldg, "sht_synthesize_adjoint")) != SHT_OK) return rc;
    if (K == 0) return SHT_OK;
    if (!ok_ptr(coeffs_bar) || !ok_ptr(grid_bar)) return fail(SHT_EINVAL, "sht_synthesize_adjoint: NULL array");
    DeviceGuard g(plan->p.device);
    cudaStream_t s = (cudaStream_t)stream;
    cudaError_t e = launch_fft_analysis(plan->p, grid_bar, ldg, K, s, false, flags & SHT_UNSCALE_COSLAT, true);
    if (e != cudaSuccess) return cuda_fail(e, "sht_synthesize_adjoint (Fourier)");
    return finish(legendre_analysis(plan->p, (float2*)coeffs_bar, ldc, K, (flags & SHT_ADD) != 0, s),
                  "sht_synthesize_adjoint (Legendre)");
}

int sht_analyze_adjoint(sht_plan* plan, const void* coeffs_bar, int64_t ldc, float* grid_bar, int64_t ldg, int K,
                        unsigned flags, void* stream) {
    int rc;
    if ((rc = check_call(plan, K, "sht_analyze_adjoint")) != SHT_OK) return rc;
    if ((rc = check_ldc(plan->p, ldc, "sht_analyze_adjoint")) != SHT_OK) return rc;
    if ((rc = check_ldg(plan->p, ldg, "sht_analyze_adjoint")) != SHT_OK) return rc;
    if (K == 0) return SHT_OK;
    if (!ok_ptr(coeffs_bar) || !ok_ptr(grid_bar)) return fail(SHT_EINVAL, "sht_analyze_adjoint: NULL array");
    DeviceGuard g(plan->p.device);
    cudaStream_t s = (cudaStream_t)stream;
    cudaError_t e = legendre_synthesis(plan->p, (const float2*)coeffs_bar, ldc, K, s);
    if (e != cudaSuccess) return cuda_fail(e, "sht_analyze_adjoint (Legendre)");
    return finish(launch_fft_synthesis(plan->p, grid_bar, ldg, K, flags & SHT_ADD, s, true),
                  "sht_analyze_adjoint (Fourier)");
}

static int ops_check(sht_plan* plan, int64_t ldc, int K, const char* what, std::initializer_list<const void*> ptrs) {
    int rc;
    if ((rc = check_call(plan, K, what)) != SHT_OK) return rc;
    if ((rc = check_ldc(plan->p, ldc, what)) != SHT_OK) return rc;
    if (K == 0) return SHT_OK;
    for (const void* q : ptrs)
        if (!q) return fail(SHT_EINVAL, "%s: NULL array", what);
    if (plan->p.nlm < 2) return fail(SHT_EINVAL, "%s: spectrum too small for operators", what);
    return SHT_OK;
}

int sht_curl(sht_plan* plan, void* out, const void* u, const void* v, int64_t ldc, int K, unsigned flags,
             double radius, void* stream) {
    int rc = ops_check(plan, ldc, K, "sht_curl", {out, u, v});
    if (rc != SHT_OK || K == 0) return rc;
    DeviceGuard g(plan->p.device);
    return finish(launch_divcurl(plan->p, (float2*)out, (const float2*)u, (const float2*)v, ldc, K, true,
                                 flags & SHT_FLIPSIGN, flags & SHT_ADD, (float)(1.0 / radius), (cudaStream_t)stream),
                  "sht_curl");
}

int sht_divergence(sht_plan* plan, void* out, const void* u, const void* v, int64_t ldc, int K, unsigned flags,
                   double radius, void* stream) {
    int rc = ops_check(plan, ldc, K, "sht_divergence", {out, u, v});
    if (rc != SHT_OK || K == 0) return rc;
    DeviceGuard g(plan->p.device);
    return finish(launch_divcurl(plan->p, (float2*)out, (const float2*)u, (const float2*)v, ldc, K, false,
                                 flags & SHT_FLIPSIGN, flags & SHT_ADD, (float)(1.0 / radius), (cudaStream_t)stream),
                  "sht_divergence");
}

int sht_uv_from_vordiv(sht_plan* plan, void* U, void* V, const void* vor, const void* div, int64_t ldc, int K,
                       double radius, void* stream) {
    int rc = ops_check(plan, ldc, K, "sht_uv_from_vordiv", {U, V, vor});
    if (rc != SHT_OK || K == 0) return rc;
    DeviceGuard g(plan->p.device);
    return finish(launch_uv_from_vordiv(plan->p, (float2*)U, (float2*)V, (const float2*)vor, (const float2*)div, ldc,
                                        K, (float)radius, (cudaStream_t)stream),
                  "sht_uv_from_vordiv");
}

int sht_laplace(sht_plan* plan, void* out, const void* alms, int64_t ldc, int K, unsigned flags, double radius,
                void* stream) {
    int rc = ops_check(plan, ldc, K, "sht_laplace", {out, alms});
    if (rc != SHT_OK || K == 0) return rc;
    DeviceGuard g(plan->p.device);
    const bool inv = flags & SHT_INVERSE;
    const double scale = radius == 1.0 ? 1.0 : (inv ? radius * radius : 1.0 / (radius * radius));
    return finish(launch_laplace(plan->p, (float2*)out, (const float2*)alms, ldc, K, inv, flags & SHT_FLIPSIGN,
                                 flags & SHT_ADD, (float)scale, (cudaStream_t)stream),
                  "sht_laplace");
}

int sht_gradient(sht_plan* plan, void* dpdx, void* dpdy, const void* p_, int64_t ldc, int K, double radius,
                 void* stream) {
    int rc = ops_check(plan, ldc, K, "sht_gradient", {dpdx, dpdy, p_});
    if (rc != SHT_OK || K == 0) return rc;
    DeviceGuard g(plan->p.device);
    return finish(launch_gradient(plan->p, (float2*)dpdx, (float2*)dpdy, (const float2*)p_, ldc, K,
                                  (float)(1.0 / radius), (cudaStream_t)stream),
                  "sht_gradient");
}

int sht_operators(sht_plan* plan, const sht_op* ops, int nops, void* stream) {
    const char* what = "sht_operators";
    if (!plan) return fail(SHT_EINVAL, "%s: plan is NULL", what);
    if (nops < 0 || nops > SHT_MAX_OPS) return fail(SHT_EINVAL, "%s: %d ops (at most %d)", what, nops, SHT_MAX_OPS);
    if (nops == 0) return SHT_OK;
    if (!ops) return fail(SHT_EINVAL, "%s: ops is NULL", what);
    const Plan& p = plan->p;
    // byte range of an array of K layers with leading dimension ldc
    auto range = [&](const void* ptr, int64_t ldc, int K) {
        const uintptr_t b = reinterpret_cast<uintptr_t>(ptr);
        return std::make_pair(b, b + (uintptr_t)(((int64_t)(K - 1) * ldc + p.nlm) * 8));
    };
    auto overlap = [](std::pair<uintptr_t, uintptr_t> x, std::pair<uintptr_t, uintptr_t> y) {
        return x.first < y.second && y.first < x.second;
    };
    struct Arr {
        const void* ptr;
        int64_t ldc;
        std::pair<uintptr_t, uintptr_t> r;
    };
    std::vector<Arr> outs, ins;
    for (int j = 0; j < nops; ++j) {
        const sht_op& o = ops[j];
        int rc = ops_check(plan, o.ldc, o.K, what, {o.out, o.a});
        if (rc != SHT_OK) return rc;
        if (o.K == 0) continue;
        const bool two_out = o.kind == SHT_OP_GRADIENT || o.kind == SHT_OP_UV_FROM_VORDIV;
        switch (o.kind) {
            case SHT_OP_CURL:
            case SHT_OP_DIVERGENCE:
                if (!o.b) return fail(SHT_EINVAL, "%s: op %d: NULL array", what, j);
                break;
            case SHT_OP_LAPLACE:
                break;
            case SHT_OP_GRADIENT:
            case SHT_OP_UV_FROM_VORDIV:
                if (!o.out2) return fail(SHT_EINVAL, "%s: op %d: NULL array", what, j);
                break;
            default:
                return fail(SHT_EINVAL, "%s: op %d: unknown kind %d", what, j, o.kind);
        }
        if (!(o.radius > 0.0)) return fail(SHT_EINVAL, "%s: op %d: radius must be positive", what, j);
        outs.push_back({o.out, o.ldc, range(o.out, o.ldc, o.K)});
        if (two_out) outs.push_back({o.out2, o.ldc, range(o.out2, o.ldc, o.K)});
        ins.push_back({o.a, o.ldc, range(o.a, o.ldc, o.K)});
        if (o.b && o.kind != SHT_OP_LAPLACE && o.kind != SHT_OP_GRADIENT) ins.push_back({o.b, o.ldc, range(o.b, o.ldc, o.K)});
    }
    for (const Arr& x : ins)
        for (const Arr& y : outs)
            if (overlap(x.r, y.r)) return fail(SHT_EINVAL, "%s: an input overlaps an output of the batch", what);
    for (size_t i = 0; i < outs.size(); ++i)
        for (size_t k = i + 1; k < outs.size(); ++k)
            if (overlap(outs[i].r, outs[k].r) && (outs[i].ptr != outs[k].ptr || outs[i].ldc != outs[k].ldc))
                return fail(SHT_EINVAL, "%s: overlapping outputs must be the same array", what);
    DeviceGuard g(p.device);
    return finish(launch_operators(p, ops, nops, (cudaStream_t)stream), what);
}

}  // extern "C"

namespace sht {
// Accessors for entry points defined in other files of the library.
const Plan* plan_impl(const sht_plan* plan) { return plan ? &plan->p : nullptr; }
int set_error(int code, const char* msg) { return fail(code, "%s", msg); }
}  // namespace sht
