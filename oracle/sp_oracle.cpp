// sp_oracle.cpp -- CPU oracle (TEST INFRASTRUCTURE ONLY; see sp_oracle.h).
//
// A restatement, in plain C++/OpenMP, of the reference's FP64 OpenMP
// execution path.  Every function cites the reference file:line it follows.
// Floating-point expressions keep the reference's operand order; the library
// is compiled with -ffp-contract=off so that each source-level operation
// rounds once, as written.
#include "sp_oracle.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <utility>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

int g_threads = 0;

// Block size of the reference's OpenMP backend (Convection.cpp:14-16).
constexpr int kBlock = 8;
// Halo width (Convection.h:13).
constexpr int kHalo = 2;

// Halo-padded field in the reference's OpenMP storage order JIK: j slowest,
// i middle, k fastest (SharedInfrastructure.h:76-80, Convection.h:19).
// Allocator whose value-initialisation is a no-op, so that a field's pages are
// first touched by the parallel zero-fill in Field::init (the threads that
// later sweep the same j-rows), not by one thread in std::vector's constructor.
template <typename T>
struct NoInitAlloc : std::allocator<T> {
    template <typename U>
    struct rebind { using other = NoInitAlloc<U>; };
    NoInitAlloc() = default;
    template <typename U>
    NoInitAlloc(const NoInitAlloc<U>&) {}
    template <typename U>
    void construct(U* p) noexcept { ::new (static_cast<void*>(p)) U; }
    template <typename U, typename... A>
    void construct(U* p, A&&... a) { ::new (static_cast<void*>(p)) U(std::forward<A>(a)...); }
};

template <typename T>
struct Field {
    int ni = 0, nj = 0, nk = 0;
    long si = 0, sj = 0;  // strides of i and j; k stride is 1
    std::vector<T, NoInitAlloc<T>> v;
    Field() = default;
    Field(int a, int b, int c) { init(a, b, c); }
    void init(int a, int b, int c) {
        ni = a; nj = b; nk = c;
        si = nk + 2 * kHalo;
        sj = (long)(ni + 2 * kHalo) * si;
        const long rows = nj + 2 * kHalo;
        v.resize((size_t)rows * sj);
        T* d = v.data();
        const long row = sj;
#pragma omp parallel for schedule(static)
        for (long j = 0; j < rows; ++j) std::fill(d + j * row, d + (j + 1) * row, T(0));
    }
    // (i,j,k) are interior coordinates; -2..n+1 address the halo.
    inline T* col(int i, int j) { return v.data() + (long)(j + kHalo) * sj + (long)(i + kHalo) * si + kHalo; }
    inline const T* col(int i, int j) const { return v.data() + (long)(j + kHalo) * sj + (long)(i + kHalo) * si + kHalo; }
    inline T& at(int i, int j, int k) { return col(i, j)[k]; }
    inline T at(int i, int j, int k) const { return col(i, j)[k]; }
};

template <typename T, typename U>
void load_dense(Field<T>& f, const U* d) {
    const int ni = f.ni, nj = f.nj, nk = f.nk;
#pragma omp parallel for schedule(static)
    for (int j = 0; j < nj; ++j)
        for (int i = 0; i < ni; ++i) {
            T* c = f.col(i, j);
            for (int k = 0; k < nk; ++k) c[k] = (T)d[((long)k * nj + j) * ni + i];
        }
}

template <typename T, typename U>
void store_dense(const Field<T>& f, U* d) {
    const int ni = f.ni, nj = f.nj, nk = f.nk;
#pragma omp parallel for schedule(static)
    for (int j = 0; j < nj; ++j)
        for (int i = 0; i < ni; ++i) {
            const T* c = f.col(i, j);
            for (int k = 0; k < nk; ++k) d[((long)k * nj + j) * ni + i] = (U)c[k];
        }
}

// Periodicity.cpp:10-135 -- I faces (interior J,K), then J (all I, interior K),
// then K (all I and J), so that edges and corners are filled too.
template <typename T>
void periodicity(Field<T>& f) {
    const int ni = f.ni, nj = f.nj, nk = f.nk;
    // ApplyPeriodicI (Periodicity.cpp:10-38)
#pragma omp parallel for schedule(static)
    for (int j = 0; j < nj; ++j)
        for (int k = 0; k < nk; ++k) {
            for (int h = 0; h < kHalo; ++h) f.at(h - kHalo, j, k) = f.at(h - kHalo + ni, j, k);
            for (int h = 0; h < kHalo; ++h) f.at(ni + h, j, k) = f.at(h, j, k);
        }
    // ApplyPeriodicJ (Periodicity.cpp:40-68)
#pragma omp parallel for schedule(static)
    for (int i = -kHalo; i < ni + kHalo; ++i)
        for (int k = 0; k < nk; ++k) {
            for (int h = 0; h < kHalo; ++h) f.at(i, h - kHalo, k) = f.at(i, h - kHalo + nj, k);
            for (int h = 0; h < kHalo; ++h) f.at(i, nj + h, k) = f.at(i, h, k);
        }
    // ApplyPeriodicK (Periodicity.cpp:70-98)
#pragma omp parallel for schedule(static)
    for (int i = -kHalo; i < ni + kHalo; ++i)
        for (int j = -kHalo; j < nj + kHalo; ++j) {
            T* c = f.col(i, j);
            for (int h = 0; h < kHalo; ++h) c[h - kHalo] = c[h - kHalo + nk];
            for (int h = 0; h < kHalo; ++h) c[nk + h] = c[h];
        }
}

// Loop over the interior in the reference's OpenMP execution model:
// 8x8 IJ blocks distributed by `omp for` (StencilOpenMP.h:224-250), the
// contiguous K column innermost.
template <typename F>
void for_blocks(int ni, int nj, F&& body) {
    const int nbi = (ni + kBlock - 1) / kBlock, nbj = (nj + kBlock - 1) / kBlock;
#pragma omp parallel for schedule(static)
    for (int b = 0; b < nbi * nbj; ++b) {
        const int bi = b % nbi, bj = b / nbi;
        const int i1 = std::min(ni, (bi + 1) * kBlock), j1 = std::min(nj, (bj + 1) * kBlock);
        for (int j = bj * kBlock; j < j1; ++j)
            for (int i = bi * kBlock; i < i1; ++i) body(i, j);
    }
}

template <typename T>
struct Params {
    T nu0, nufreq, cx, cy, cz, dx, dx2;
    bool upwind;
};

// RHS4Stage (Convection.cpp:57-82) with Advection4 (ConvectionFunctions.h:66-104)
// and Laplace4 (ConvectionFunctions.h:135-167).
template <typename T>
void rhs4(const Field<T>& q, Field<T>& k, const Params<T>& P, T nu) {
    const int nk = q.nk;
    const long si = q.si, sj = q.sj;
    const T one = 1, eight = 8, twelve = 12, sixteen = 16, thirty = 30;
    for_blocks(q.ni, q.nj, [&](int i, int j) {
        const T* c = q.col(i, j);
        T* o = k.col(i, j);
        for (int kk = 0; kk < nk; ++kk) {
            const T* p = c + kk;
            T dq_di = -one * p[-2 * si] + eight * p[-si] - eight * p[si] + one * p[2 * si];
            T dq_dj = -one * p[-2 * sj] + eight * p[-sj] - eight * p[sj] + one * p[2 * sj];
            T dq_dk = -one * p[-2] + eight * p[-1] - eight * p[1] + one * p[2];
            T tensadv = (P.cx * dq_di + P.cy * dq_dj + P.cz * dq_dk) / (twelve * P.dx);
            T d2q_di2 = -one * p[-2 * si] + sixteen * p[-si] - thirty * p[0] + sixteen * p[si] - one * p[2 * si];
            T d2q_dj2 = -one * p[-2 * sj] + sixteen * p[-sj] - thirty * p[0] + sixteen * p[sj] - one * p[2 * sj];
            T d2q_dk2 = -one * p[-2] + sixteen * p[-1] - thirty * p[0] + sixteen * p[1] - one * p[2];
            T tenslapl = nu * ((d2q_di2 + d2q_dj2 + d2q_dk2) / (twelve * P.dx2));
            o[kk] = tensadv + tenslapl;
        }
    });
}

// RHS2Stage (Convection.cpp:30-55) with Advection2 (ConvectionFunctions.h:4-64,
// the UPWINDADVECTION branch when P.upwind, CMakeLists.txt:101-105) and
// Laplace2 (ConvectionFunctions.h:106-132).
template <typename T>
void rhs2(const Field<T>& q, Field<T>& k, const Params<T>& P, T nu) {
    const int nk = q.nk;
    const long si = q.si, sj = q.sj;
    const T one = 1, two = 2, zero = 0;
    for_blocks(q.ni, q.nj, [&](int i, int j) {
        const T* c = q.col(i, j);
        T* o = k.col(i, j);
        for (int kk = 0; kk < nk; ++kk) {
            const T* p = c + kk;
            T tensadv;
            if (P.upwind) {
                T dq_di = P.cx > zero ? (p[0] - p[-si]) : (p[si] - p[0]);
                T dq_dj = P.cy > zero ? (p[0] - p[-sj]) : (p[sj] - p[0]);
                T dq_dk = P.cz > zero ? (p[0] - p[-1]) : (p[1] - p[0]);
                tensadv = -(P.cx * dq_di + P.cy * dq_dj + P.cz * dq_dk) / P.dx;
            } else {
                T dq_di = one * p[-si] - one * p[si];
                T dq_dj = one * p[-sj] - one * p[sj];
                T dq_dk = one * p[-1] - one * p[1];
                tensadv = (P.cx * dq_di + P.cy * dq_dj + P.cz * dq_dk) / (two * P.dx);
            }
            T d2q_di2 = one * p[-si] - two * p[0] + one * p[si];
            T d2q_dj2 = one * p[-sj] - two * p[0] + one * p[sj];
            T d2q_dk2 = one * p[-1] - two * p[0] + one * p[1];
            T tenslapl = nu * ((d2q_di2 + d2q_dj2 + d2q_dk2) / P.dx2);
            o[kk] = tensadv + tenslapl;
        }
    });
}

// EulerStage (Convection.cpp:84-101): qeulerout = qmainin + dt*k.
template <typename T>
void euler_stage(const Field<T>& qmainin, const Field<T>& k, T dt, Field<T>& qeulerout) {
    const int nk = k.nk;
    for_blocks(k.ni, k.nj, [&](int i, int j) {
        const T* a = qmainin.col(i, j);
        const T* b = k.col(i, j);
        T* o = qeulerout.col(i, j);
        for (int kk = 0; kk < nk; ++kk) o[kk] = a[kk] + dt * b[kk];
    });
}

// RKStage (Convection.cpp:103-127): qout = qin + dt/6*(k1 + 2k2 + 2k3 + k4).
template <typename T>
void rk_stage(const Field<T>& qin, const Field<T>& k1, const Field<T>& k2, const Field<T>& k3,
              const Field<T>& k4, T dt, Field<T>& qout) {
    const int nk = k1.nk;
    const T two = 2, six = 6;
    for_blocks(k1.ni, k1.nj, [&](int i, int j) {
        const T* a = qin.col(i, j);
        const T* b1 = k1.col(i, j);
        const T* b2 = k2.col(i, j);
        const T* b3 = k3.col(i, j);
        const T* b4 = k4.col(i, j);
        T* o = qout.col(i, j);
        for (int kk = 0; kk < nk; ++kk)
            o[kk] = a[kk] + dt / six * (b1[kk] + two * b2[kk] + two * b3[kk] + b4[kk]);
    });
}

// The propagator: class Convection (Convection.h:22-108, Convection.cpp:131-392).
template <typename T>
struct Convection {
    Params<T> P;
    Field<T> qInternal, k1, k2, k3, k4;  // Convection.cpp:159-163

    Convection(const orc_params& p) {
        P.nu0 = (T)p.nu0; P.nufreq = (T)p.nufreq;
        P.cx = (T)p.cx; P.cy = (T)p.cy; P.cz = (T)p.cz;
        P.dx = (T)p.dx; P.dx2 = P.dx * P.dx;  // Convection.cpp:134
        P.upwind = p.upwind != 0;
        qInternal.init(p.ni, p.nj, p.nk);
        k1.init(p.ni, p.nj, p.nk); k2.init(p.ni, p.nj, p.nk);
        k3.init(p.ni, p.nj, p.nk); k4.init(p.ni, p.nj, p.nk);
    }

    // computenu (Convection.h:81-84); evaluated in double as the reference does.
    T computenu(double t) const { return (T)((double)P.nu0 * (1. + .5 * std::sin((double)P.nufreq * t))); }

    // DoRK4Timestep (Convection.cpp:318-370).
    void rk4_step(Field<T>& in, Field<T>& out, double t, double dt) {
        const T dthalf = (T)(dt * .5);
        const T nu = computenu(t);
        periodicity(in);                       // halo of the input, in place
        rhs4(in, k1, P, nu);                   // k1 = RHS(in)
        euler_stage(in, k1, dthalf, qInternal);
        periodicity(qInternal);
        rhs4(qInternal, k2, P, nu);
        euler_stage(in, k2, dthalf, qInternal);
        periodicity(qInternal);
        rhs4(qInternal, k3, P, nu);
        euler_stage(in, k3, (T)dt, qInternal);
        periodicity(qInternal);
        rhs4(qInternal, k4, P, nu);
        rk_stage(in, k1, k2, k3, k4, (T)dt, out);
    }

    // DoEulerTimestep (Convection.cpp:372-392).
    void euler_step(Field<T>& in, Field<T>& out, double t, double dt) {
        const T nu = computenu(t);
        periodicity(in);
        rhs2(in, k1, P, nu);
        euler_stage(in, k1, (T)dt, out);
    }

    // DoRK4 (Convection.cpp:292-303): step 0 in->out, then out->out in place.
    void DoRK4(Field<T>& in, Field<T>& out, double tStart, double dt, int n) {
        if (n > 0) rk4_step(in, out, tStart, dt);
        int i = 0;
        for (--n; n > 0; --n) rk4_step(out, out, tStart + (++i) * dt, dt);
    }

    // DoEuler (Convection.cpp:305-316).
    void DoEuler(Field<T>& in, Field<T>& out, double tStart, double dt, int n) {
        if (n > 0) euler_step(in, out, tStart, dt);
        int i = 0;
        for (--n; n > 0; --n) euler_step(out, out, tStart + (++i) * dt, dt);
    }
};

bool valid(const orc_params* p) {
    return p && p->ni >= 2 && p->nj >= 2 && p->nk >= 2 && p->dx > 0;
}

template <typename T>
int run_prop(const orc_params* p, const T* in, T* out, double tStart, double dt, int n, bool rk) {
    if (!valid(p) || !in || !out || n < 0) return -1;
    if (n == 0) return 0;  // DoRK4/DoEuler with 0 steps leave the output untouched
    Convection<T> c(*p);
    Field<T> fin(p->ni, p->nj, p->nk), fout(p->ni, p->nj, p->nk);
    load_dense(fin, in);
    if (rk) c.DoRK4(fin, fout, tStart, dt, n);
    else c.DoEuler(fin, fout, tStart, dt, n);
    store_dense(fout, out);
    return 0;
}

// RuntimeConfiguration.cpp:133-151 (round totals up to a multiple of the slice
// count) and RuntimeConfiguration.h:54-101 (derived values).
struct Derived {
    int tsFineTot, tsCoarseTot, tsF, tsC;
    double dtF, dtC, slice;
};
bool derive(const orc_parareal_cfg* c, Derived* d) {
    if (!c || c->timeSlices < 1 || c->timeStepsFine < 1 || c->timeStepsCoarse < 1 || c->kmax < 0 ||
        !(c->endTime > 0))
        return false;
    const int P = c->timeSlices;
    int f = c->timeStepsFine, g = c->timeStepsCoarse;
    if (f % P != 0) f = (f / P + 1) * P;
    if (g % P != 0) g = (g / P + 1) * P;
    d->tsFineTot = f; d->tsCoarseTot = g;
    d->tsF = f / P; d->tsC = g / P;
    d->dtF = c->endTime / f;
    d->dtC = c->endTime / g;
    d->slice = c->endTime / P;
    return true;
}

// The coarse propagator G used by the Parareal oracle.  Its state is stored in
// FP64 (EULER_F64, RK4_F64) or FP32 (RK4_F32, EULER_F32).
struct Coarse {
    int kind;
    Convection<double> c64;
    Convection<float> c32;
    Field<float> t32a;
    Coarse(const orc_params& p, int k) : kind(k), c64(p), c32(p) {
        if (kind == ORC_COARSE_RK4_F32 || kind == ORC_COARSE_EULER_F32) t32a.init(p.ni, p.nj, p.nk);
    }
    bool f32() const { return kind == ORC_COARSE_RK4_F32 || kind == ORC_COARSE_EULER_F32; }
    // out = G^n(in) in the coarse precision; in and out are FP64 fields (for the
    // FP32 kinds the input is rounded to FP32 and the output widened back).
    void prop64(Field<double>& in, Field<double>& out, double t0, double dt, int n) {
        if (n == 0) { if (&in != &out) out.v = in.v; return; }
        if (!f32()) {
            if (kind == ORC_COARSE_EULER_F64) c64.DoEuler(in, out, t0, dt, n);
            else c64.DoRK4(in, out, t0, dt, n);
            return;
        }
        for (size_t i = 0; i < in.v.size(); ++i) t32a.v[i] = (float)in.v[i];
        if (kind == ORC_COARSE_EULER_F32) c32.DoEuler(t32a, t32a, t0, dt, n);
        else c32.DoRK4(t32a, t32a, t0, dt, n);
        for (size_t i = 0; i < in.v.size(); ++i) out.v[i] = (double)t32a.v[i];
    }
};

double err_maxrel_field(const Field<double>& f, const Field<double>& r) {
    // computeErrorReference (main.cpp:98-139)
    double error = 0., maxfield = 0.;
    for (int j = 0; j < f.nj; ++j)
        for (int i = 0; i < f.ni; ++i) {
            const double* a = f.col(i, j);
            const double* b = r.col(i, j);
            for (int k = 0; k < f.nk; ++k) {
                error = std::max(error, std::abs(a[k] - b[k]));
                maxfield = std::max(std::abs(a[k]), maxfield);
            }
        }
    return error / maxfield;
}

double err_l2rel_field(const Field<double>& f, const Field<double>& r) {
    double num = 0., den = 0.;
    for (int j = 0; j < f.nj; ++j)
        for (int i = 0; i < f.ni; ++i) {
            const double* a = f.col(i, j);
            const double* b = r.col(i, j);
            for (int k = 0; k < f.nk; ++k) {
                const double d = a[k] - b[k];
                num += d * d;
                den += b[k] * b[k];
            }
        }
    return std::sqrt(num / den);
}

// ---------------------------------------------------------------------------
// Adjoint helpers.  R(q) = sum_d c_d D_d q + nu L q with D_d and L the
// Advection4 / Laplace4 stencils (ConvectionFunctions.h:66-104,135-167).
// The transpose is applied by mirroring the stencil offsets.
struct Star13 {
    // weights of the 13-point star: w0 centre, wx[o], wy[o], wz[o] for o = -2..2
    double w0, wx[5], wy[5], wz[5];
};

Star13 star_R(const Params<double>& P, double nu) {
    Star13 s;
    const double a = 1. / (12. * P.dx), l = nu / (12. * P.dx2);
    const double adv[5] = {-1., 8., 0., -8., 1.};
    const double lap[5] = {-1., 16., -30., 16., -1.};
    for (int o = 0; o < 5; ++o) {
        s.wx[o] = P.cx * adv[o] * a + lap[o] * l;
        s.wy[o] = P.cy * adv[o] * a + lap[o] * l;
        s.wz[o] = P.cz * adv[o] * a + lap[o] * l;
    }
    s.w0 = 0.;
    return s;
}

// out = S^T in, for the star S: (S^T m)[x] = sum_o w_o m[x - o].
void apply_transpose(const Star13& s, Field<double>& m, Field<double>& out) {
    periodicity(m);
    const long si = m.si, sj = m.sj;
    const int nk = m.nk;
    for_blocks(m.ni, m.nj, [&](int i, int j) {
        const double* c = m.col(i, j);
        double* o = out.col(i, j);
        for (int kk = 0; kk < nk; ++kk) {
            const double* p = c + kk;
            double acc = 0.;
            for (int t = 0; t < 5; ++t) {
                const int off = t - 2;
                acc += s.wx[t] * p[-off * si] + s.wy[t] * p[-off * sj] + s.wz[t] * p[-off];
            }
            o[kk] = acc;
        }
    });
}

// Per-axis derivative stencils applied to y: dx[d] = D_d y, lap = L y.
void partials(Field<double>& y, const Params<double>& P, Field<double>& dxo, Field<double>& dyo,
              Field<double>& dzo, Field<double>& lo) {
    periodicity(y);
    const long si = y.si, sj = y.sj;
    const int nk = y.nk;
    for_blocks(y.ni, y.nj, [&](int i, int j) {
        const double* c = y.col(i, j);
        double *ox = dxo.col(i, j), *oy = dyo.col(i, j), *oz = dzo.col(i, j), *ol = lo.col(i, j);
        for (int kk = 0; kk < nk; ++kk) {
            const double* p = c + kk;
            const double di = -p[-2 * si] + 8. * p[-si] - 8. * p[si] + p[2 * si];
            const double dj = -p[-2 * sj] + 8. * p[-sj] - 8. * p[sj] + p[2 * sj];
            const double dk = -p[-2] + 8. * p[-1] - 8. * p[1] + p[2];
            const double li = -p[-2 * si] + 16. * p[-si] - 30. * p[0] + 16. * p[si] - p[2 * si];
            const double lj = -p[-2 * sj] + 16. * p[-sj] - 30. * p[0] + 16. * p[sj] - p[2 * sj];
            const double lk = -p[-2] + 16. * p[-1] - 30. * p[0] + 16. * p[1] - p[2];
            ox[kk] = di / (12. * P.dx);
            oy[kk] = dj / (12. * P.dx);
            oz[kk] = dk / (12. * P.dx);
            ol[kk] = (li + lj + lk) / (12. * P.dx2);
        }
    });
}

double dot_interior(const Field<double>& a, const Field<double>& b) {
    double s = 0.;
    for (int j = 0; j < a.nj; ++j)
        for (int i = 0; i < a.ni; ++i) {
            const double* x = a.col(i, j);
            const double* y = b.col(i, j);
            for (int k = 0; k < a.nk; ++k) s += x[k] * y[k];
        }
    return s;
}

}  // namespace

extern "C" {

void orc_set_threads(int n) {
    g_threads = n;
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#endif
}

int orc_get_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

int orc_rk4(const orc_params* p, const double* in, double* out, double tStart, double dt, int n) {
    return run_prop<double>(p, in, out, tStart, dt, n, true);
}
int orc_euler(const orc_params* p, const double* in, double* out, double tStart, double dt, int n) {
    return run_prop<double>(p, in, out, tStart, dt, n, false);
}
int orc_rk4_f32(const orc_params* p, const float* in, float* out, double tStart, double dt, int n) {
    return run_prop<float>(p, in, out, tStart, dt, n, true);
}
int orc_euler_f32(const orc_params* p, const float* in, float* out, double tStart, double dt, int n) {
    return run_prop<float>(p, in, out, tStart, dt, n, false);
}

int orc_rhs4(const orc_params* p, const double* q, double* k, double t) {
    if (!valid(p) || !q || !k) return -1;
    Convection<double> c(*p);
    Field<double> f(p->ni, p->nj, p->nk), o(p->ni, p->nj, p->nk);
    load_dense(f, q);
    periodicity(f);
    rhs4(f, o, c.P, c.computenu(t));
    store_dense(o, k);
    return 0;
}

int orc_rhs2(const orc_params* p, const double* q, double* k, double t) {
    if (!valid(p) || !q || !k) return -1;
    Convection<double> c(*p);
    Field<double> f(p->ni, p->nj, p->nk), o(p->ni, p->nj, p->nk);
    load_dense(f, q);
    periodicity(f);
    rhs2(f, o, c.P, c.computenu(t));
    store_dense(o, k);
    return 0;
}

int orc_periodicity_jik(int ni, int nj, int nk, double* field) {
    if (ni < 1 || nj < 1 || nk < 1 || !field) return -1;
    Field<double> f(ni, nj, nk);
    std::memcpy(f.v.data(), field, f.v.size() * sizeof(double));
    periodicity(f);
    std::memcpy(field, f.v.data(), f.v.size() * sizeof(double));
    return 0;
}

struct orc_rk4_session {
    Convection<double> c;
    Field<double> fin, fout;
    explicit orc_rk4_session(const orc_params& p) : c(p), fin(p.ni, p.nj, p.nk), fout(p.ni, p.nj, p.nk) {}
};

orc_rk4_session* orc_rk4_session_create(const orc_params* p, const double* in) {
    if (!valid(p) || !in) return nullptr;
    orc_rk4_session* s = new orc_rk4_session(*p);
    load_dense(s->fin, in);
    return s;
}

int orc_rk4_session_run(orc_rk4_session* s, double tStart, double dt, int n) {
    if (!s || n < 0) return -1;
    s->c.DoRK4(s->fin, s->fout, tStart, dt, n);
    return 0;
}

int orc_rk4_session_result(const orc_rk4_session* s, double* out) {
    if (!s || !out) return -1;
    store_dense(s->fout, out);
    return 0;
}

void orc_rk4_session_destroy(orc_rk4_session* s) { delete s; }

int orc_parareal_derived(const orc_parareal_cfg* c, int out[4], double dout[3]) {
    Derived d;
    if (!derive(c, &d)) return -1;
    out[0] = d.tsFineTot; out[1] = d.tsCoarseTot; out[2] = d.tsF; out[3] = d.tsC;
    dout[0] = d.dtF; dout[1] = d.dtC; dout[2] = d.slice;
    return 0;
}

int orc_parareal(const orc_params* p, const orc_parareal_cfg* c, const double* q0, double* q_out,
                 double* q_serial, double* err_max, double* err_l2) {
    return orc_parareal_ex(p, c, q0, q_out, q_serial, err_max, err_l2, nullptr, nullptr);
}

int orc_parareal_ex(const orc_params* p, const orc_parareal_cfg* c, const double* q0, double* q_out,
                    double* q_serial, double* err_max, double* err_l2, double* defect, double* q_iters) {
    Derived d;
    if (!valid(p) || !derive(c, &d) || !q0 || !q_out) return -1;
    if (c->coarse < 0 || c->coarse > 3) return -1;
    const int P = c->timeSlices;
    Convection<double> fine(*p);
    Coarse coarse(*p, c->coarse);

    // Parareal::DoSerial (Parareal.h:250-253)
    Field<double> qref(p->ni, p->nj, p->nk);
    {
        Field<double> qin(p->ni, p->nj, p->nk);
        load_dense(qin, q0);
        fine.DoRK4(qin, qref, 0., d.dtF, d.tsF * P);
        if (d.tsF * P == 0) qref.v = qin.v;
    }
    if (q_serial) store_dense(qref, q_serial);

    // One "rank" per slice (Parareal.h:48-108): qinitial (U), q (result),
    // qfine, qcoarseold, qcoarsenew.
    std::vector<Field<double>> U(P), Q(P), Fq(P), Gold(P), Gnew(P);
    for (int r = 0; r < P; ++r) {
        U[r].init(p->ni, p->nj, p->nk);
        load_dense(U[r], q0);
        Q[r].init(p->ni, p->nj, p->nk);
        Fq[r].init(p->ni, p->nj, p->nk);
        Gold[r].init(p->ni, p->nj, p->nk);
        Gnew[r].init(p->ni, p->nj, p->nk);
    }
    // Predictor (Parareal.h:113-114): U_r = G^{tsC*r}(q0) from t=0, then Gold = G(U_r).
    for (int r = 0; r < P; ++r) {
        const double tStart = d.slice * r;  // main.cpp:157
        coarse.prop64(U[r], U[r], 0., d.dtC, d.tsC * r);
        coarse.prop64(U[r], Gold[r], tStart, d.dtC, d.tsC);
    }
    // Slice-end values before iteration 1 (for the defect of iteration 1): the
    // predictor's U_{r+1}, and G(U_{P-1}) at the last slice's end.
    std::vector<Field<double>> Qprev;
    if (defect) {
        Qprev.resize(P);
        for (int r = 0; r < P; ++r) Qprev[r].v = (r + 1 < P ? U[r + 1].v : Gold[P - 1].v);
        for (int r = 0; r < P; ++r) {
            Qprev[r].ni = p->ni; Qprev[r].nj = p->nj; Qprev[r].nk = p->nk;
            Qprev[r].si = U[0].si; Qprev[r].sj = U[0].sj;
        }
    }
    // Per iteration: the defect max_r ||Q_r^k - Q_r^{k-1}||_2 / ||Q_r^k||_2 over
    // the slice ends, and the last slice's result as a dense field.
    const long ncell = (long)p->ni * p->nj * p->nk;
    auto record = [&](int k) {
        if (err_max) err_max[k] = err_maxrel_field(Q[P - 1], qref);
        if (err_l2) err_l2[k] = err_l2rel_field(Q[P - 1], qref);
        if (q_iters) store_dense(Q[P - 1], q_iters + (size_t)k * ncell);
        if (defect) {
            double dm = 0.;
            for (int r = 0; r < P; ++r) {
                double num = 0., den = 0.;
                for (int j = 0; j < p->nj; ++j)
                    for (int i = 0; i < p->ni; ++i) {
                        const double* a = Q[r].col(i, j);
                        const double* b = Qprev[r].col(i, j);
                        for (int kk = 0; kk < p->nk; ++kk) {
                            const double e = a[kk] - b[kk];
                            num += e * e;
                            den += a[kk] * a[kk];
                        }
                    }
                if (den > 0) dm = std::max(dm, std::sqrt(num / den));
                Qprev[r].v = Q[r].v;
            }
            defect[k] = dm;
        }
    };
    // Increment form of the correction: U_{r+1} = F(U_r^old) + G(U_r^new - U_r^old).
    // G is linear (linear PDE), so this equals the reference's
    // G(U_r^new) + F(U_r^old) - G(U_r^old) in exact arithmetic.
    if (c->coarse_delta) {
        Field<double> delta(p->ni, p->nj, p->nk), gd(p->ni, p->nj, p->nk);
        for (int k = 0; k < c->kmax; ++k) {
            for (int r = 0; r < P; ++r) {
                const double tStart = d.slice * r;
                const double tStartFine = tStart + d.dtF;
                if (c->async && r != 0) {
                    fine.DoRK4(U[r], Fq[r], tStart, d.dtF, 1);
                    fine.DoRK4(Fq[r], Fq[r], tStartFine, d.dtF, d.tsF - 1);
                } else {
                    fine.DoRK4(U[r], Fq[r], tStart, d.dtF, d.tsF);
                }
                if (r != 0) {
                    for (size_t i = 0; i < delta.v.size(); ++i) delta.v[i] = Q[r - 1].v[i] - U[r].v[i];
                    U[r].v = Q[r - 1].v;
                } else {
                    std::fill(delta.v.begin(), delta.v.end(), 0.);
                }
                coarse.prop64(delta, gd, tStart, d.dtC, d.tsC);
                for (size_t i = 0; i < gd.v.size(); ++i) Q[r].v[i] = Fq[r].v[i] + gd.v[i];
            }
            record(k);
        }
        store_dense(Q[P - 1], q_out);
        return 0;
    }
    // Iterations (Parareal.h:116-165), the rank pipeline executed slice by slice.
    for (int k = 0; k < c->kmax; ++k) {
        for (int r = 0; r < P; ++r) {
            const double tStart = d.slice * r;
            const double tStartFine = tStart + d.dtF;  // Parareal.h:107
            if (c->async && r != 0) {
                fine.DoRK4(U[r], Fq[r], tStart, d.dtF, 1);
                fine.DoRK4(Fq[r], Fq[r], tStartFine, d.dtF, d.tsF - 1);
            } else {
                fine.DoRK4(U[r], Fq[r], tStart, d.dtF, d.tsF);
            }
            if (r != 0) U[r].v = Q[r - 1].v;  // receive U_r^{k+1} from rank r-1
            coarse.prop64(U[r], Gnew[r], tStart, d.dtC, d.tsC);
            // UpdateStage (Parareal.h:19-35): q = qcoarsenew + qfine - qcoarseold
            {
                Field<double>& q = Q[r];
                const Field<double>& gn = Gnew[r];
                const Field<double>& fq = Fq[r];
                const Field<double>& go = Gold[r];
                const int nk = q.nk;
                for_blocks(q.ni, q.nj, [&](int i, int j) {
                    const double* a = gn.col(i, j);
                    const double* b = fq.col(i, j);
                    const double* e = go.col(i, j);
                    double* o = q.col(i, j);
                    for (int kk = 0; kk < nk; ++kk) o[kk] = a[kk] + b[kk] - e[kk];
                });
            }
            std::swap(Gold[r].v, Gnew[r].v);  // qcoarseold.SwapWith(qcoarsenew)
        }
        record(k);
    }
    store_dense(Q[P - 1], q_out);
    return 0;
}

int orc_adjoint_rk4(const orc_params* p, const double* q0, const double* q_target, double tStart,
                    double dt, int n, double* J, double* grad_q0, double* grad_par) {
    if (!valid(p) || !q0 || !q_target || n < 0) return -1;
    Convection<double> c(*p);
    const int ni = p->ni, nj = p->nj, nk = p->nk;
    std::vector<Field<double>> qs(n + 1);
    for (auto& f : qs) f.init(ni, nj, nk);
    load_dense(qs[0], q0);
    for (int s = 0; s < n; ++s) c.DoRK4(qs[s], qs[s + 1], tStart + s * dt, dt, 1);
    // DoRK4 steps at t = tStart + s*dt (Convection.cpp:301-302).
    Field<double> tgt(ni, nj, nk);
    load_dense(tgt, q_target);
    Field<double> lam(ni, nj, nk);
    double jv = 0.;
    for (size_t i = 0; i < lam.v.size(); ++i) lam.v[i] = 0.;
    for (int j = 0; j < nj; ++j)
        for (int i = 0; i < ni; ++i)
            for (int k = 0; k < nk; ++k) {
                const double d = qs[n].at(i, j, k) - tgt.at(i, j, k);
                jv += 0.5 * d * d;
                lam.at(i, j, k) = d;
            }
    double gnu0 = 0., gcx = 0., gcy = 0., gcz = 0.;
    Field<double> y[4], mu(ni, nj, nk), g(ni, nj, nk), kk(ni, nj, nk), lam_new(ni, nj, nk);
    Field<double> Dx(ni, nj, nk), Dy(ni, nj, nk), Dz(ni, nj, nk), L(ni, nj, nk);
    for (auto& f : y) f.init(ni, nj, nk);
    const double a_stage[4] = {0., .5, .5, 1.};  // y_{s+1} = q + h*a*k_s
    const double b[4] = {1. / 6., 1. / 3., 1. / 3., 1. / 6.};
    for (int s = n - 1; s >= 0; --s) {
        const double t = tStart + s * dt;
        const double nu = c.computenu(t);
        const double dnu = 1. + .5 * std::sin(p->nufreq * t);  // d nu / d nu0
        // Recompute the stage inputs y_1..y_4 of step s.
        y[0].v = qs[s].v;
        for (int st = 0; st < 3; ++st) {
            periodicity(y[st]);
            rhs4(y[st], kk, c.P, nu);
            const double h = dt * a_stage[st + 1];
            for (size_t i = 0; i < kk.v.size(); ++i) y[st + 1].v[i] = qs[s].v[i] + h * kk.v[i];
        }
        const Star13 S = star_R(c.P, nu);
        lam_new.v = lam.v;
        Field<double> gbar_next;  // ybar_{s+1}
        bool have_next = false;
        Field<double> ybar(ni, nj, nk);
        for (int st = 3; st >= 0; --st) {
            // mu_s = h b_s lam + h a_{s+1,s} ybar_{s+1}
            for (size_t i = 0; i < mu.v.size(); ++i) {
                double v = dt * b[st] * lam.v[i];
                if (have_next) v += dt * a_stage[st + 1] * ybar.v[i];
                mu.v[i] = v;
            }
            // parameter gradient: mu_s^T dR/dtheta (y_s)
            partials(y[st], c.P, Dx, Dy, Dz, L);
            gnu0 += dnu * dot_interior(mu, L);
            gcx += dot_interior(mu, Dx);
            gcy += dot_interior(mu, Dy);
            gcz += dot_interior(mu, Dz);
            // ybar_s = R^T mu_s
            apply_transpose(S, mu, ybar);
            for (size_t i = 0; i < ybar.v.size(); ++i) lam_new.v[i] += ybar.v[i];
            have_next = true;
        }
        // Halo entries of lam_new carry garbage from the halo of ybar; only the
        // interior is meaningful.  Keep the interior.
        lam.v = lam_new.v;
    }
    if (J) *J = jv;
    if (grad_q0) store_dense(lam, grad_q0);
    if (grad_par) { grad_par[0] = gnu0; grad_par[1] = gcx; grad_par[2] = gcy; grad_par[3] = gcz; }
    return 0;
}

double orc_exactq(double nu0, double nufreq, double cx, double cy, double cz, double x, double y,
                  double z, double t) {
    // exactQ (ConvectionSolution.h:8-20), with the reference's value of pi.
    const double pi = 3.14159265358979;
    const double a = nufreq > 0 ? nu0 * t - (nu0 / (2. * nufreq)) * (std::cos(nufreq * t) - 1.) : nu0 * t;
    return std::sin(2. * pi * (x - cx * t)) * std::sin(2. * pi * (y - cy * t)) *
           std::sin(2. * pi * (z - cz * t)) * std::exp(-12. * pi * pi * a);
}

int orc_fillq(const orc_params* p, double t, double* q) {
    // fillQ on [0,1]^3 (ConvectionSolution.h:23-52, called at main.cpp:214).
    if (!valid(p) || !q) return -1;
    const double dxhalf = 1. / p->ni / 2., dyhalf = 1. / p->nj / 2., dzhalf = 1. / p->nk / 2.;
    for (int i = 0; i < p->ni; ++i)
        for (int j = 0; j < p->nj; ++j)
            for (int k = 0; k < p->nk; ++k) {
                const double x = 0. + (2 * i + 1) * dxhalf;
                const double y = 0. + (2 * j + 1) * dyhalf;
                const double z = 0. + (2 * k + 1) * dzhalf;
                q[((long)k * p->nj + j) * p->ni + i] =
                    orc_exactq(p->nu0, p->nufreq, p->cx, p->cy, p->cz, x, y, z, t);
            }
    return 0;
}

double orc_error_maxrel(const double* f, const double* r, long n) {
    double error = 0., maxfield = 0.;
    for (long i = 0; i < n; ++i) {
        error = std::max(error, std::abs(f[i] - r[i]));
        maxfield = std::max(std::abs(f[i]), maxfield);
    }
    return error / maxfield;
}

double orc_error_l2rel(const double* f, const double* r, long n) {
    double num = 0., den = 0.;
    for (long i = 0; i < n; ++i) {
        const double d = f[i] - r[i];
        num += d * d;
        den += r[i] * r[i];
    }
    return std::sqrt(num / den);
}

}  // extern "C"
