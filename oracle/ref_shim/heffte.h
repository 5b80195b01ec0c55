/*
 * Single-rank stand-in for the part of heFFTe's interface the reference
 * solver uses (heFFTe v2.4, dependency of the reference through
 * src/domain.h:4-9 and src/fourier_transform.h:12-51).
 *
 * Test infrastructure only.  heFFTe and FFTW are not installed here, so this
 * header supplies box3d<>, fft3d_r2c<backend>, scale::{none,full} and a
 * project-written FP64 mixed-radix Stockham FFT (radices 2,3,4,5,8 plus a
 * direct DFT for other primes).  Semantics follow heFFTe's documented
 * contract for a 2-D R2C transform on one rank:
 *   - physical layout: x fastest, Nx*Ny reals per field (Nz = 1);
 *   - spectral layout: x fastest, (Nx/2+1)*Ny complex per field
 *     (r2c direction 0, as in Domain2D::R2C_DIRECTION);
 *   - forward is unnormalised, backward with scale::full divides by Nx*Ny;
 *   - batch fields are contiguous, one after another;
 *   - a C2R ignores the imaginary parts of the kx = 0 and kx = Nx/2 entries
 *     (FFTW's c2r convention for Hermitian input);
 *   - rows and columns are split over host threads (SHHD_REF_THREADS, default
 *     all hardware threads), the shared-memory counterpart of heFFTe's rank
 *     decomposition.
 */
#ifndef SHHD_ORACLE_SHIM_HEFFTE_H
#define SHHD_ORACLE_SHIM_HEFFTE_H

#include <mpi.h>

#include <algorithm>
#include <array>
#include <cmath>
#include <complex>
#include <cstddef>
#include <cstdlib>
#include <stdexcept>
#include <thread>
#include <vector>

namespace shimfft {

using cplx = std::complex<double>;

// Threads for the transforms: SHHD_REF_THREADS, else all hardware threads.
inline int num_threads() {
    static const int n = [] {
        if (const char* e = std::getenv("SHHD_REF_THREADS")) {
            const int v = std::atoi(e);
            if (v > 0) return v;
        }
        const unsigned h = std::thread::hardware_concurrency();
        return h > 0 ? static_cast<int>(h) : 1;
    }();
    return n;
}

// fn(begin, end) over [0, n) split into contiguous chunks, one per thread.
template <typename F>
void parallel_for(int n, F&& fn) {
    const int t = std::min(num_threads(), std::max(1, n));
    if (t <= 1) {
        fn(0, n);
        return;
    }
    std::vector<std::thread> pool;
    pool.reserve(static_cast<std::size_t>(t - 1));
    const int chunk = (n + t - 1) / t;
    for (int i = 1; i < t; ++i) {
        const int b = i * chunk, e = std::min(n, b + chunk);
        if (b < e) pool.emplace_back([&fn, b, e] { fn(b, e); });
    }
    fn(0, std::min(n, chunk));
    for (auto& th : pool) th.join();
}

// One complex FFT plan of length n (Stockham autosort, out of place ping-pong).
class Plan {
    int n_ = 0;
    std::vector<int> radices_;
    // per stage: twiddles w^(q*k) for k < p, q < R, sign -1
    std::vector<std::vector<cplx>> tw_;

public:
    explicit Plan(int n) : n_(n) {
        if (n <= 0) throw std::runtime_error("shim fft: length must be positive");
        int m = n;
        for (int r : {8, 4, 2, 3, 5}) {
            while (m % r == 0) { radices_.push_back(r); m /= r; }
        }
        for (int p = 7; m > 1; p += 2) {
            while (m % p == 0) { radices_.push_back(p); m /= p; }
        }
        int p = 1;
        for (int R : radices_) {
            std::vector<cplx> t(static_cast<std::size_t>(p) * R);
            for (int k = 0; k < p; ++k) {
                for (int q = 0; q < R; ++q) {
                    const double ang = -2.0 * M_PI * double(q) * double(k) / double(p * R);
                    t[static_cast<std::size_t>(k) * R + q] = cplx(std::cos(ang), std::sin(ang));
                }
            }
            tw_.push_back(std::move(t));
            p *= R;
        }
    }

    int size() const { return n_; }

    // In-place transform of x (length n); sign = -1 forward, +1 backward; work has length n.
    void execute(cplx* x, cplx* work, int sign) const {
        cplx* src = x;
        cplx* dst = work;
        int p = 1;
        for (std::size_t s = 0; s < radices_.size(); ++s) {
            const int R = radices_[s];
            const int m = n_ / R;
            const cplx* t = tw_[s].data();
            cplx v[64];
            cplx V[64];
            for (int i = 0; i < m; ++i) {
                const int k = i % p;
                for (int q = 0; q < R; ++q) {
                    cplx w = t[static_cast<std::size_t>(k) * R + q];
                    if (sign > 0) w = std::conj(w);
                    v[q] = src[i + q * m] * w;
                }
                dft(R, v, V, sign);
                const int base = (i - k) * R + k;
                for (int r = 0; r < R; ++r) dst[base + r * p] = V[r];
            }
            std::swap(src, dst);
            p *= R;
        }
        if (src != x) {
            for (int i = 0; i < n_; ++i) x[i] = src[i];
        }
    }

private:
    static void dft(int R, const cplx* v, cplx* V, int sign) {
        const double s = static_cast<double>(sign);
        if (R == 2) {
            V[0] = v[0] + v[1];
            V[1] = v[0] - v[1];
            return;
        }
        if (R == 4) {
            const cplx a = v[0] + v[2], b = v[0] - v[2];
            const cplx c = v[1] + v[3], d = (v[1] - v[3]) * cplx(0.0, s);
            V[0] = a + c; V[2] = a - c; V[1] = b + d; V[3] = b - d;
            return;
        }
        if (R == 8) {
            cplx e[4], o[4], E[4], O[4];
            for (int j = 0; j < 4; ++j) { e[j] = v[2 * j]; o[j] = v[2 * j + 1]; }
            dft(4, e, E, sign);
            dft(4, o, O, sign);
            const double h = std::sqrt(0.5);
            const cplx w[4] = {cplx(1.0, 0.0), cplx(h, s * h), cplx(0.0, s), cplx(-h, s * h)};
            for (int j = 0; j < 4; ++j) {
                const cplx t = O[j] * w[j];
                V[j] = E[j] + t;
                V[j + 4] = E[j] - t;
            }
            return;
        }
        for (int r = 0; r < R; ++r) {
            cplx acc(0.0, 0.0);
            for (int q = 0; q < R; ++q) {
                const double ang = s * 2.0 * M_PI * double((q * r) % R) / double(R);
                acc += v[q] * cplx(std::cos(ang), std::sin(ang));
            }
            V[r] = acc;
        }
    }
};

} // namespace shimfft

namespace heffte {

template <typename index = int>
struct box3d {
    std::array<index, 3> low{{0, 0, 0}};
    std::array<index, 3> high{{-1, -1, -1}};
    std::array<index, 3> size{{0, 0, 0}};

    box3d() = default;
    box3d(std::array<index, 3> l, std::array<index, 3> h) : low(l), high(h) {
        for (int d = 0; d < 3; ++d) size[d] = high[d] - low[d] + 1;
    }
    bool empty() const { return size[0] <= 0 || size[1] <= 0 || size[2] <= 0; }
    index count() const { return empty() ? 0 : size[0] * size[1] * size[2]; }
};

enum class scale { none, full, symmetric };

namespace backend {
struct fftw {};
struct mkl {};
} // namespace backend

template <typename backend_tag, typename index = int>
class fft3d_r2c {
    int nx_ = 0;
    int ny_ = 0;
    int hx_ = 0;  // nx/2 + 1
    shimfft::Plan px_;
    shimfft::Plan py_;

public:
    fft3d_r2c(box3d<index> inbox, box3d<index> outbox, int r2c_direction, MPI_Comm)
        : nx_(inbox.size[0]), ny_(inbox.size[1]), hx_(inbox.size[0] / 2 + 1), px_(inbox.size[0]), py_(inbox.size[1]) {
        if (r2c_direction != 0) throw std::runtime_error("shim heffte: only r2c direction 0 is supported");
        if (inbox.low[0] != 0 || inbox.low[1] != 0 || inbox.size[2] != 1)
            throw std::runtime_error("shim heffte: single-rank 2-D boxes only");
        if (outbox.size[0] != hx_ || outbox.size[1] != ny_)
            throw std::runtime_error("shim heffte: spectral box must be (nx/2+1) x ny");
    }

    index size_inbox() const { return nx_ * ny_; }
    index size_outbox() const { return hx_ * ny_; }

    void forward(int batch, const double* in, std::complex<double>* out, scale s) const {
        for (int b = 0; b < batch; ++b) {
            forward_one(in + static_cast<std::size_t>(b) * nx_ * ny_, out + static_cast<std::size_t>(b) * hx_ * ny_);
            if (s == scale::full) scale_by(out + static_cast<std::size_t>(b) * hx_ * ny_, 1.0 / (double(nx_) * ny_));
        }
    }

    void backward(int batch, const std::complex<double>* in, double* out, scale s) const {
        for (int b = 0; b < batch; ++b) {
            double* o = out + static_cast<std::size_t>(b) * nx_ * ny_;
            backward_one(in + static_cast<std::size_t>(b) * hx_ * ny_, o);
            if (s == scale::full) {
                const double f = 1.0 / (double(nx_) * ny_);
                for (int i = 0; i < nx_ * ny_; ++i) o[i] *= f;
            }
        }
    }

private:
    void scale_by(std::complex<double>* x, double f) const {
        for (int i = 0; i < hx_ * ny_; ++i) x[i] *= f;
    }

    // rows (x) real->complex two at a time, then columns (y) complex forward;
    // rows and columns are independent, so OpenMP threads split them
    void forward_one(const double* in, std::complex<double>* out) const {
        shimfft::parallel_for((ny_ + 1) / 2, [&](int p0, int p1) {
            std::vector<shimfft::cplx> z(nx_), w(nx_);
            for (int y = 2 * p0; y < std::min(ny_, 2 * p1); y += 2) {
                const bool pair = (y + 1 < ny_);
                for (int x = 0; x < nx_; ++x)
                    z[x] = shimfft::cplx(in[y * nx_ + x], pair ? in[(y + 1) * nx_ + x] : 0.0);
                px_.execute(z.data(), w.data(), -1);
                for (int k = 0; k < hx_; ++k) {
                    const shimfft::cplx a = z[k];
                    const shimfft::cplx b = std::conj(z[(nx_ - k) % nx_]);
                    out[y * hx_ + k] = 0.5 * (a + b);
                    if (pair) out[(y + 1) * hx_ + k] = shimfft::cplx(0.0, -0.5) * (a - b);
                }
            }
        });
        shimfft::parallel_for(hx_, [&](int k0, int k1) {
            std::vector<shimfft::cplx> col(ny_), wc(ny_);
            for (int k = k0; k < k1; ++k) {
                for (int y = 0; y < ny_; ++y) col[y] = out[y * hx_ + k];
                py_.execute(col.data(), wc.data(), -1);
                for (int y = 0; y < ny_; ++y) out[y * hx_ + k] = col[y];
            }
        });
    }

    // columns (y) complex backward, then rows (x) complex->real two at a time
    void backward_one(const std::complex<double>* in, double* out) const {
        std::vector<shimfft::cplx> mid(static_cast<std::size_t>(hx_) * ny_);
        const bool even = (nx_ % 2 == 0);
        shimfft::parallel_for(hx_, [&](int k0, int k1) {
            std::vector<shimfft::cplx> col(ny_), wc(ny_);
            for (int k = k0; k < k1; ++k) {
                for (int y = 0; y < ny_; ++y) col[y] = in[y * hx_ + k];
                py_.execute(col.data(), wc.data(), +1);
                for (int y = 0; y < ny_; ++y) mid[static_cast<std::size_t>(y) * hx_ + k] = col[y];
            }
        });
        shimfft::parallel_for((ny_ + 1) / 2, [&](int p0, int p1) {
            std::vector<shimfft::cplx> z(nx_), w(nx_);
            for (int y = 2 * p0; y < std::min(ny_, 2 * p1); y += 2) {
                const bool pair = (y + 1 < ny_);
                const shimfft::cplx* r0 = &mid[static_cast<std::size_t>(y) * hx_];
                const shimfft::cplx* r1 = pair ? &mid[static_cast<std::size_t>(y + 1) * hx_] : nullptr;
                for (int k = 0; k < nx_; ++k) z[k] = 0.0;
                for (int k = 0; k < hx_; ++k) {
                    shimfft::cplx a = r0[k];
                    shimfft::cplx b = pair ? r1[k] : shimfft::cplx(0.0, 0.0);
                    const bool self_conjugate = (k == 0) || (even && k == nx_ / 2);
                    if (self_conjugate) {
                        a = shimfft::cplx(a.real(), 0.0);
                        b = shimfft::cplx(b.real(), 0.0);
                        z[k] = a + shimfft::cplx(0.0, 1.0) * b;
                    } else {
                        z[k] = a + shimfft::cplx(0.0, 1.0) * b;
                        z[nx_ - k] = std::conj(a) + shimfft::cplx(0.0, 1.0) * std::conj(b);
                    }
                }
                px_.execute(z.data(), w.data(), +1);
                for (int x = 0; x < nx_; ++x) {
                    out[y * nx_ + x] = z[x].real();
                    if (pair) out[(y + 1) * nx_ + x] = z[x].imag();
                }
            }
        });
    }
};

} // namespace heffte

#endif
