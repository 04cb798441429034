// sep-CMA-ES and dd-CMA-ES, ask/tell form. Formulas and update order follow
// ta3_trainer/src/pagmo/sep_cmaes.cpp:92-279 and ta3_trainer/src/pagmo/dd_cmaes.cpp:100-358;
// linear algebra is written out over std::vector (no Eigen here).
#include "cmaes.hpp"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <sstream>
#include <stdexcept>

namespace ta3b::host {

// ------------------------------------------------------------------ eigensolver

bool sym_eig(Mat const& A, vec& w, Mat* V) {
    int const n = A.n;
    Mat a = A;
    Mat v(n, 1.0);
    w.assign(size_t(n), 0.0);
    double norm_all = 0.0;
    for (double x : a.a) norm_all += x * x;
    bool ok = false;
    for (int sweep = 0; sweep < 100; ++sweep) {
        double off = 0.0;
        for (int p = 0; p < n; ++p)
            for (int q = p + 1; q < n; ++q) off += a(p, q) * a(p, q);
        if (off <= 1e-30 * norm_all || off == 0.0) {
            ok = true;
            break;
        }
        for (int p = 0; p < n; ++p) {
            for (int q = p + 1; q < n; ++q) {
                double const apq = a(p, q);
                if (apq == 0.0) continue;
                // rotation angle annihilating a(p,q) (Golub & Van Loan, symmetric Schur)
                double const theta = (a(q, q) - a(p, p)) / (2.0 * apq);
                double const t = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
                double const c = 1.0 / std::sqrt(t * t + 1.0);
                double const s = t * c;
                for (int k = 0; k < n; ++k) {          // A <- A J (columns p, q)
                    double const akp = a(k, p), akq = a(k, q);
                    a(k, p) = c * akp - s * akq;
                    a(k, q) = s * akp + c * akq;
                }
                for (int k = 0; k < n; ++k) {          // A <- J^T A (rows p, q)
                    double const apk = a(p, k), aqk = a(q, k);
                    a(p, k) = c * apk - s * aqk;
                    a(q, k) = s * apk + c * aqk;
                }
                a(p, q) = a(q, p) = 0.0;
                if (V)
                    for (int k = 0; k < n; ++k) {
                        double const vkp = v(k, p), vkq = v(k, q);
                        v(k, p) = c * vkp - s * vkq;
                        v(k, q) = s * vkp + c * vkq;
                    }
            }
        }
    }
    for (int i = 0; i < n; ++i) w[size_t(i)] = a(i, i);
    if (V) *V = v;
    return ok;
}

namespace {

double sq_norm(double const* x, int n) {
    double s = 0.0;
    for (int i = 0; i < n; ++i) s += x[i] * x[i];
    return s;
}

// y = M x
void mat_vec(Mat const& m, double const* x, double* y) {
    int const n = m.n;
    for (int i = 0; i < n; ++i) {
        double s = 0.0;
        double const* row = &m.a[size_t(i) * n];
        for (int j = 0; j < n; ++j) s += row[j] * x[j];
        y[i] = s;
    }
}

// sorted candidate order (lessF), over all k or the best `keep`
std::vector<int> rank(int k, double const* f, int keep) {
    std::vector<int> order(static_cast<size_t>(k));
    std::iota(order.begin(), order.end(), 0);
    auto const cmp = [f](int a, int b) { return less_f(f[a], f[b]); };
    if (keep < k)
        std::partial_sort(order.begin(), order.begin() + keep, order.end(), cmp);
    else
        std::sort(order.begin(), order.end(), cmp);
    return order;
}

// ---- binary state blobs: magic, kind, then length-prefixed fields
constexpr char kMagic[8] = {'T', 'A', '3', 'C', 'M', 'A', 'E', 'S'};
constexpr uint32_t kVersion = 1;

struct Writer {
    std::string out;
    void raw(void const* p, size_t n) { out.append(static_cast<char const*>(p), n); }
    template<class T> void pod(T v) { raw(&v, sizeof v); }
    void doubles(vec const& v) {
        pod<uint64_t>(v.size());
        raw(v.data(), v.size() * sizeof(double));
    }
    void text(std::string const& s) {
        pod<uint64_t>(s.size());
        raw(s.data(), s.size());
    }
};

struct Reader {
    std::string const& in;
    size_t pos;
    bool ok = true;
    bool raw(void* p, size_t n) {
        if (!ok || pos + n > in.size()) return ok = false;
        std::memcpy(p, in.data() + pos, n);
        pos += n;
        return true;
    }
    template<class T> T pod() {
        T v{};
        raw(&v, sizeof v);
        return v;
    }
    vec doubles() {
        uint64_t const n = pod<uint64_t>();
        if (!ok || n > (in.size() - pos) / sizeof(double)) {
            ok = false;
            return {};
        }
        vec v(n);
        raw(v.data(), n * sizeof(double));
        return v;
    }
    std::string text() {
        uint64_t const n = pod<uint64_t>();
        if (!ok || n > in.size() - pos) {
            ok = false;
            return {};
        }
        std::string s(in.data() + pos, n);
        pos += n;
        return s;
    }
};

std::string rng_text(std::mt19937 const& rng, std::normal_distribution<double> const& nd) {
    std::ostringstream os;
    os.precision(17);
    os << rng << ' ' << nd;
    return os.str();
}

bool rng_from_text(std::string const& s, std::mt19937& rng, std::normal_distribution<double>& nd) {
    std::istringstream is(s);
    is >> rng >> nd;
    return !is.fail();
}

void header(Writer& w, CmaKind kind, int n) {
    w.raw(kMagic, sizeof kMagic);
    w.pod<uint32_t>(kVersion);
    w.pod<uint32_t>(uint32_t(kind));
    w.pod<uint32_t>(uint32_t(n));
}

} // namespace

Cma* Cma::load(std::string const& blob, std::string* err) {
    auto fail = [err](char const* m) -> Cma* {
        if (err) *err = m;
        return nullptr;
    };
    if (blob.size() < sizeof kMagic + 12 || std::memcmp(blob.data(), kMagic, sizeof kMagic) != 0)
        return fail("not a CMA-ES state blob");
    uint32_t version, kind;
    std::memcpy(&version, blob.data() + 8, 4);
    std::memcpy(&kind, blob.data() + 12, 4);
    if (version != kVersion) return fail("unsupported CMA-ES state version");
    if (kind == uint32_t(CmaKind::SEP)) {
        auto* c = new SepCma();
        if (c->restore(blob, 16)) return c;
        delete c;
        return fail("corrupt sep-CMA-ES state");
    }
    if (kind == uint32_t(CmaKind::DD)) {
        auto* c = new DdCma();
        if (c->restore(blob, 16)) return c;
        delete c;
        return fail("corrupt dd-CMA-ES state");
    }
    return fail("unknown CMA-ES kind");
}

// ------------------------------------------------------------------ sep-CMA-ES

SepCma::SepCma(vec const& x0, vec const& lb, vec const& ub, double sigma0, uint32_t seed) {
    if (!(sigma0 > 0.0)) throw std::invalid_argument("sigma0 must be positive");
    n_ = int(x0.size());
    rng_.seed(seed);
    // sep_cmaes.cpp:78-89: sigma = sigma0, diag = box width^2, paths zero
    sigma_ = sigma0;
    mean_ = x0;
    diag_.resize(static_cast<size_t>(n_));
    for (int j = 0; j < n_; ++j) diag_[size_t(j)] = std::pow(std::max(ub[size_t(j)] - lb[size_t(j)], 1e-6), 2);
    pc_.assign(size_t(n_), 0.0);
    ps_.assign(size_t(n_), 0.0);
}

vec SepCma::axis_std() const {
    vec s(static_cast<size_t>(n_));
    for (int j = 0; j < n_; ++j) s[size_t(j)] = sigma_ * std::sqrt(diag_[size_t(j)]);
    return s;
}

void SepCma::whiten(int k, double const* x, double* z) const {
    // ask: x = m + sigma * sqrt(diag) * z
    vec const s = axis_std();
    for (int i = 0; i < k; ++i)
        for (int j = 0; j < n_; ++j)
            z[size_t(i) * n_ + j] = (x[size_t(i) * n_ + j] - mean_[size_t(j)]) / s[size_t(j)];
}

void SepCma::ask(int lam, double* out) {
    // sep_cmaes.cpp:170-178: per candidate, n normal draws, x = m + sigma * sqrt(diag) * z
    axis_.resize(static_cast<size_t>(n_));
    for (int j = 0; j < n_; ++j) axis_[size_t(j)] = std::sqrt(diag_[size_t(j)]);
    z_.resize(size_t(lam) * n_);
    x_.resize(size_t(lam) * n_);
    for (int i = 0; i < lam; ++i) {
        double* z = &z_[size_t(i) * n_];
        double* x = &x_[size_t(i) * n_];
        for (int j = 0; j < n_; ++j) z[j] = normal_(rng_);
        for (int j = 0; j < n_; ++j) x[j] = mean_[size_t(j)] + sigma_ * (axis_[size_t(j)] * z[j]);
    }
    double dx = 0.0;
    if (lam > 0)
        for (int j = 0; j < n_; ++j) {
            double const s = sigma_ * (axis_[size_t(j)] * z_[size_t(lam - 1) * n_ + j]);
            dx += s * s;
        }
    last_dx_ = std::sqrt(dx);
    std::memcpy(out, x_.data(), x_.size() * sizeof(double));
    asked_ = lam;
}

void SepCma::tell(int k, int const* idx, double const* fitness) {
    int const lam = k;
    int const mu = lam / 2;
    double const n = n_;
    // sep_cmaes.cpp:123-139: weights over the mu best, learning rates
    vec w(static_cast<size_t>(mu));
    for (int i = 0; i < mu; ++i) w[size_t(i)] = std::log(double(mu) + 0.5) - std::log(double(i) + 1.0);
    double const wsum = std::accumulate(w.begin(), w.end(), 0.0);
    for (double& x : w) x /= wsum;
    double const mu_eff = 1.0 / sq_norm(w.data(), mu);
    double const boost = (n + 2.0) / 3.0;
    double const cc = (4.0 + mu_eff / n) / (n + 4.0 + 2.0 * mu_eff / n);
    double const cs = (mu_eff + 2.0) / (n + mu_eff + 5.0);
    double const c1 = std::min(1.0, boost * 2.0 / ((n + 1.3) * (n + 1.3) + mu_eff));
    double const cmu = std::min(1.0 - c1, boost * 2.0 * (mu_eff - 2.0 + 1.0 / mu_eff) / ((n + 2.0) * (n + 2.0) + mu_eff));
    double const damps = 1.0 + 2.0 * std::max(0.0, std::sqrt((mu_eff - 1.0) / (n + 1.0)) - 1.0) + cs;
    double const chi_n = std::sqrt(n) * (1.0 - 1.0 / (4.0 * n) + 1.0 / (21.0 * n * n));
    count_eval_ += uint64_t(lam);

    // sep_cmaes.cpp:243-257: elite steps y_i = (x_i:lam - m) / sigma, yw = y w, m += sigma yw
    std::vector<int> const order = rank(k, fitness, mu);
    std::vector<double> y(size_t(mu) * n_);
    vec yw(size_t(n_), 0.0);
    for (int i = 0; i < mu; ++i) {
        int const c = idx ? idx[order[size_t(i)]] : order[size_t(i)];
        double const* x = &x_[size_t(c) * n_];
        for (int j = 0; j < n_; ++j) y[size_t(i) * n_ + j] = (x[j] - mean_[size_t(j)]) / sigma_;
    }
    for (int j = 0; j < n_; ++j) {
        double s = 0.0;
        for (int i = 0; i < mu; ++i) s += y[size_t(i) * n_ + j] * w[size_t(i)];
        yw[size_t(j)] = s;
    }
    for (int j = 0; j < n_; ++j) mean_[size_t(j)] += sigma_ * yw[size_t(j)];

    // sep_cmaes.cpp:259-264: paths; C^(-1/2) is the per-axis division
    double const fs = std::sqrt(cs * (2.0 - cs) * mu_eff);
    for (int j = 0; j < n_; ++j) ps_[size_t(j)] = (1.0 - cs) * ps_[size_t(j)] + fs * (yw[size_t(j)] / axis_[size_t(j)]);
    double const ps2 = sq_norm(ps_.data(), n_);
    double const hsig =
        ps2 / n / (1.0 - std::pow(1.0 - cs, 2.0 * double(count_eval_) / double(lam))) < 2.0 + 4.0 / (n + 1.0);
    double const fc = hsig * std::sqrt(cc * (2.0 - cc) * mu_eff);
    for (int j = 0; j < n_; ++j) pc_[size_t(j)] = (1.0 - cc) * pc_[size_t(j)] + fc * yw[size_t(j)];

    // sep_cmaes.cpp:267-273: diagonal rank-one + rank-mu, floor, then sigma
    for (int j = 0; j < n_; ++j) {
        double rmu = 0.0;
        for (int i = 0; i < mu; ++i) {
            double const v = y[size_t(i) * n_ + j];
            rmu += v * v * w[size_t(i)];
        }
        double const dj = diag_[size_t(j)];
        double const pcj = pc_[size_t(j)];
        double const v = (1.0 - c1 - cmu) * dj + c1 * (pcj * pcj + (1.0 - hsig) * cc * (2.0 - cc) * dj) + cmu * rmu;
        diag_[size_t(j)] = std::max(v, 1e-20);
    }
    sigma_ *= std::exp(std::min(0.6, cs / damps * (std::sqrt(ps2) / chi_n - 1.0)));
}

std::string SepCma::save() const {
    Writer w;
    header(w, CmaKind::SEP, n_);
    w.pod<double>(sigma_);
    w.pod<uint64_t>(count_eval_);
    w.doubles(mean_);
    w.doubles(diag_);
    w.doubles(pc_);
    w.doubles(ps_);
    w.text(rng_text(rng_, normal_));
    return w.out;
}

bool SepCma::restore(std::string const& blob, size_t pos) {
    Reader r{blob, pos};
    n_ = int(r.pod<uint32_t>());
    sigma_ = r.pod<double>();
    count_eval_ = r.pod<uint64_t>();
    mean_ = r.doubles();
    diag_ = r.doubles();
    pc_ = r.doubles();
    ps_ = r.doubles();
    std::string const t = r.text();
    if (!r.ok || !rng_from_text(t, rng_, normal_)) return false;
    size_t const n = size_t(n_);
    return mean_.size() == n && diag_.size() == n && pc_.size() == n && ps_.size() == n;
}

// ------------------------------------------------------------------ dd-CMA-ES

namespace {
constexpr double kBetaThresh = 2.0;   // dd_cmaes.cpp:23
constexpr double kExpo = 0.75;        // dd_cmaes.cpp:149

// dd_cmaes.cpp:129-166: every constant that depends on (n, lambda)
struct DdConsts {
    int n_pos = 0;
    vec w, wc, wd;
    double mu_eff_pos = 0, mu_eff_neg = 0, cs = 0, ds = 0, chi_n = 0, cone = 0, cmu = 0, cc = 0, cdone = 0, cdmu = 0,
           cdc = 0;
    uint64_t teig = 1;

    DdConsts(int dim, int lam) {
        double const n = dim;
        w.resize(size_t(lam));
        for (int i = 0; i < lam; ++i) w[size_t(i)] = std::log((double(lam) + 1.0) / 2.0) - std::log(double(i) + 1.0);
        n_pos = int(std::count_if(w.begin(), w.end(), [](double x) { return x > 0.0; }));
        double sp = 0.0, sn = 0.0;
        for (int i = 0; i < n_pos; ++i) sp += w[size_t(i)];
        for (int i = n_pos; i < lam; ++i) sn += w[size_t(i)];
        for (int i = 0; i < n_pos; ++i) w[size_t(i)] /= sp;
        for (int i = n_pos; i < lam; ++i) w[size_t(i)] /= std::fabs(sn);
        mu_eff_pos = 1.0 / sq_norm(w.data(), n_pos);
        mu_eff_neg = 1.0 / sq_norm(w.data() + n_pos, lam - n_pos);
        double const mp = mu_eff_pos;
        cs = (mp + 2.0) / (n + mp + 5.0);
        ds = 1.0 + cs + 2.0 * std::max(0.0, std::sqrt((mp - 1.0) / (n + 1.0)) - 1.0);
        chi_n = std::sqrt(n) * (1.0 - 1.0 / (4.0 * n) + 1.0 / (21.0 * n * n));
        double const mu_prime = mp + 1.0 / mp - 2.0 + double(lam) / (2.0 * double(lam) + 10.0);
        cone = 1.0 / (2.0 * ((n + 1.0) / 2.0 + 1.0) * std::pow(n + 1.0, kExpo) + mp / 2.0);
        cmu = std::min(1.0 - cone, mu_prime * cone);
        cc = std::sqrt(mp * cone) / 2.0;
        cdone = 1.0 / (4.0 * std::pow(n + 1.0, kExpo) + mp / 2.0);
        cdmu = std::min(1.0 - cdone, mu_prime * cdone);
        cdc = std::sqrt(mp * cdone) / 2.0;
        double const neg_limit = 1.0 + 2.0 * mu_eff_neg / (mp + 2.0);
        wc = w;
        wd = w;
        double const fc = std::min(1.0 + cone / cmu, neg_limit);
        double const fd = std::min(1.0 + cdone / cdmu, neg_limit);
        for (int i = n_pos; i < lam; ++i) {
            wc[size_t(i)] *= fc;
            wd[size_t(i)] *= fd;
        }
        double const beta_eig = 10.0 * n;
        teig = std::max<unsigned long long>(1, static_cast<unsigned long long>(1.0 / (beta_eig * (cone + cmu))));
    }
};
} // namespace

DdCma::DdCma(vec const& x0, vec const& lb, vec const& ub, double sigma0, uint32_t seed, bool active) {
    if (!(sigma0 > 0.0)) throw std::invalid_argument("sigma0 must be positive");
    n_ = int(x0.size());
    active_ = active;
    rng_.seed(seed);
    // dd_cmaes.cpp:74-97: sigma0 folded into D (per-axis std = sigma0 * box width), C = I
    sigma_ = 1.0;
    mean_ = x0;
    d_.resize(static_cast<size_t>(n_));
    for (int j = 0; j < n_; ++j) d_[size_t(j)] = sigma0 * std::max(ub[size_t(j)] - lb[size_t(j)], 1e-6);
    corr_ = Mat(n_, 1.0);
    sqrt_c_ = Mat(n_, 1.0);
    inv_sqrt_c_ = Mat(n_, 1.0);
    acc_ = Mat(n_, 0.0);
    sqrt_eig_.assign(size_t(n_), 1.0);
    pc_.assign(size_t(n_), 0.0);
    pdc_.assign(size_t(n_), 0.0);
    ps_.assign(size_t(n_), 0.0);
}

vec DdCma::axis_std() const {
    vec s(static_cast<size_t>(n_));
    for (int j = 0; j < n_; ++j) s[size_t(j)] = sigma_ * d_[size_t(j)] * std::sqrt(corr_(j, j));
    return s;
}

void DdCma::whiten(int k, double const* x, double* z) const {
    // ask: x = m + (sigma d) * sqrtC z, so z = C^(-1/2) ((x - m) / (sigma d))
    vec y(static_cast<size_t>(n_));
    for (int i = 0; i < k; ++i) {
        for (int j = 0; j < n_; ++j)
            y[size_t(j)] = (x[size_t(i) * n_ + j] - mean_[size_t(j)]) / (sigma_ * d_[size_t(j)]);
        mat_vec(inv_sqrt_c_, y.data(), z + size_t(i) * n_);
    }
}

void DdCma::ask(int lam, double* out) {
    // dd_cmaes.cpp:205-213: z column by column, y = sqrtC z, x = m + (sigma d) * y
    z_.resize(size_t(lam) * n_);
    y_.resize(size_t(lam) * n_);
    for (int i = 0; i < lam; ++i)
        for (int j = 0; j < n_; ++j) z_[size_t(i) * n_ + j] = normal_(rng_);
    vec scale(static_cast<size_t>(n_));
    for (int j = 0; j < n_; ++j) scale[size_t(j)] = sigma_ * d_[size_t(j)];
    for (int i = 0; i < lam; ++i) {
        double* y = &y_[size_t(i) * n_];
        mat_vec(sqrt_c_, &z_[size_t(i) * n_], y);
        double* x = out + size_t(i) * n_;
        for (int j = 0; j < n_; ++j) x[j] = y[j] * scale[size_t(j)] + mean_[size_t(j)];
    }
    double dx = 0.0;
    if (lam > 0)
        for (int j = 0; j < n_; ++j) {
            double const s = scale[size_t(j)] * y_[size_t(lam - 1) * n_ + j];
            dx += s * s;
        }
    last_dx_ = std::sqrt(dx);
    asked_ = lam;
}

void DdCma::tell(int k, int const* idx, double const* fitness) {
    int const lam = k;
    double const n = n_;
    DdConsts const K(n_, lam);
    int const np = K.n_pos, nr = lam - np;

    // dd_cmaes.cpp:279-283: rank all evaluated candidates, z in fitness order
    std::vector<int> const order = rank(k, fitness, k);
    std::vector<double> zs(size_t(lam) * n_);
    for (int i = 0; i < lam; ++i) {
        int const c = idx ? idx[order[size_t(i)]] : order[size_t(i)];
        std::memcpy(&zs[size_t(i) * n_], &z_[size_t(c) * n_], size_t(n_) * sizeof(double));
    }
    auto Z = [&](int i, int j) { return zs[size_t(i) * n_ + j]; };

    // 7: recombination (cm = 1)
    vec dz(size_t(n_), 0.0), dy(static_cast<size_t>(n_)), ddy(static_cast<size_t>(n_));
    for (int i = 0; i < np; ++i)
        for (int j = 0; j < n_; ++j) dz[size_t(j)] += Z(i, j) * K.w[size_t(i)];
    mat_vec(sqrt_c_, dz.data(), dy.data());
    for (int j = 0; j < n_; ++j) {
        ddy[size_t(j)] = d_[size_t(j)] * dy[size_t(j)];
        mean_[size_t(j)] += sigma_ * ddy[size_t(j)];
    }

    // 8: step size, exact cumulation normaliser
    double const cs = K.cs;
    ps_factor_ = (1.0 - cs) * (1.0 - cs) * ps_factor_ + cs * (2.0 - cs);
    double const fs = std::sqrt(cs * (2.0 - cs) * K.mu_eff_pos);
    for (int j = 0; j < n_; ++j) ps_[size_t(j)] = (1.0 - cs) * ps_[size_t(j)] + fs * dz[size_t(j)];
    double const ps2 = sq_norm(ps_.data(), n_);
    double const hsig = ps2 / ps_factor_ / n < 2.0 + 4.0 / (n + 1.0);
    sigma_ *= std::exp((std::sqrt(ps2) / K.chi_n - std::sqrt(ps_factor_)) * cs / K.ds);

    // 9: accumulate the C update in z-space
    Mat rank_upd(n_, 0.0);
    double id_coef = 0.0;
    for (int i = 0; i < np; ++i) {
        double const wi = K.w[size_t(i)];
        id_coef += wi;
        for (int a = 0; a < n_; ++a) {
            double const za = wi * Z(i, a);
            for (int b = 0; b < n_; ++b) rank_upd(a, b) += za * Z(i, b);
        }
    }
    vec neg_w(static_cast<size_t>(nr));
    if (active_) {
        for (int i = 0; i < nr; ++i) neg_w[size_t(i)] = K.wc[size_t(np + i)] * n / sq_norm(&zs[size_t(np + i) * n_], n_);
        for (int i = 0; i < nr; ++i) {
            double const wi = neg_w[size_t(i)];
            for (int a = 0; a < n_; ++a) {
                double const za = wi * Z(np + i, a);
                for (int b = 0; b < n_; ++b) rank_upd(a, b) += za * Z(np + i, b);
            }
        }
        for (int i = np; i < lam; ++i) id_coef += K.wc[size_t(i)];
    }
    double const cc = K.cc;
    double const fcc = hsig * std::sqrt(cc * (2.0 - cc) * K.mu_eff_pos);
    for (int j = 0; j < n_; ++j) pc_[size_t(j)] = (1.0 - cc) * pc_[size_t(j)] + fcc * ddy[size_t(j)];
    pc_factor_ = (1.0 - cc) * (1.0 - cc) * pc_factor_ + hsig * cc * (2.0 - cc);
    vec q(static_cast<size_t>(n_)), zp(static_cast<size_t>(n_));
    for (int j = 0; j < n_; ++j) q[size_t(j)] = pc_[size_t(j)] / d_[size_t(j)];
    mat_vec(inv_sqrt_c_, q.data(), zp.data());
    for (int a = 0; a < n_; ++a)
        for (int b = 0; b < n_; ++b) acc_(a, b) += K.cmu * rank_upd(a, b) + K.cone * (zp[size_t(a)] * zp[size_t(b)]);
    for (int a = 0; a < n_; ++a) acc_(a, a) -= K.cmu * id_coef + K.cone * pc_factor_;

    // 10: D with the fast rate, damped by beta when C is far from I
    double const cdc = K.cdc;
    double const fdc = hsig * std::sqrt(cdc * (2.0 - cdc) * K.mu_eff_pos);
    for (int j = 0; j < n_; ++j) pdc_[size_t(j)] = (1.0 - cdc) * pdc_[size_t(j)] + fdc * ddy[size_t(j)];
    pdc_factor_ = (1.0 - cdc) * (1.0 - cdc) * pdc_factor_ + hsig * cdc * (2.0 - cdc);
    for (int j = 0; j < n_; ++j) q[size_t(j)] = pdc_[size_t(j)] / d_[size_t(j)];
    mat_vec(inv_sqrt_c_, q.data(), zp.data());
    vec d_upd(static_cast<size_t>(n_));
    for (int j = 0; j < n_; ++j) d_upd[size_t(j)] = K.cdone * (zp[size_t(j)] * zp[size_t(j)] - pdc_factor_);
    for (int j = 0; j < n_; ++j) {
        double s = 0.0;
        for (int i = 0; i < np; ++i) s += Z(i, j) * Z(i, j) * K.wd[size_t(i)];
        d_upd[size_t(j)] += K.cdmu * s;
    }
    if (active_) {
        for (int i = 0; i < nr; ++i) neg_w[size_t(i)] = K.wd[size_t(np + i)] * n / sq_norm(&zs[size_t(np + i) * n_], n_);
        for (int j = 0; j < n_; ++j) {
            double s = 0.0;
            for (int i = 0; i < nr; ++i) s += Z(np + i, j) * Z(np + i, j) * neg_w[size_t(i)];
            d_upd[size_t(j)] += K.cdmu * s;
        }
        double const wd_sum = std::accumulate(K.wd.begin(), K.wd.end(), 0.0);
        for (double& v : d_upd) v -= K.cdmu * wd_sum;
    } else {
        double const wd_pos = std::accumulate(K.wd.begin(), K.wd.begin() + np, 0.0);
        for (double& v : d_upd) v -= K.cdmu * wd_pos;
    }
    double const emax = *std::max_element(sqrt_eig_.begin(), sqrt_eig_.end());
    double const emin = *std::min_element(sqrt_eig_.begin(), sqrt_eig_.end());
    double const beta = 1.0 / std::max(1.0, emax / emin - kBetaThresh + 1.0);
    for (int j = 0; j < n_; ++j) d_[size_t(j)] *= std::exp(beta / 2.0 * d_upd[size_t(j)]);

    // 11: apply the accumulated update to C every teig generations
    ++t_;
    if (t_ % K.teig == 0) {
        vec ev;
        sym_eig(acc_, ev, nullptr);
        double const min_eig = *std::min_element(ev.begin(), ev.end());
        double const fac = std::min(0.75 / std::fabs(min_eig), 1.0);
        // C = sqrtC (I + fac Z) sqrtC
        Mat m(n_, 1.0), tmp(n_, 0.0), c(n_, 0.0);
        for (size_t i = 0; i < m.a.size(); ++i) m.a[i] += fac * acc_.a[i];
        for (int i = 0; i < n_; ++i)
            for (int kk = 0; kk < n_; ++kk) {
                double const s = sqrt_c_(i, kk);
                for (int j = 0; j < n_; ++j) tmp(i, j) += s * m(kk, j);
            }
        for (int i = 0; i < n_; ++i)
            for (int kk = 0; kk < n_; ++kk) {
                double const s = tmp(i, kk);
                for (int j = 0; j < n_; ++j) c(i, j) += s * sqrt_c_(kk, j);
            }
        // back to a correlation matrix: its variances move into d
        vec cd(static_cast<size_t>(n_));
        for (int j = 0; j < n_; ++j) {
            cd[size_t(j)] = std::sqrt(c(j, j));
            d_[size_t(j)] *= cd[size_t(j)];
        }
        for (int i = 0; i < n_; ++i)
            for (int j = 0; j < n_; ++j) c(i, j) = c(i, j) / cd[size_t(i)] / cd[size_t(j)];
        for (int i = 0; i < n_; ++i)
            for (int j = 0; j < n_; ++j) corr_(i, j) = (c(i, j) + c(j, i)) / 2.0;
        vec lam_c;
        Mat v;
        if (sym_eig(corr_, lam_c, &v)) {
            for (int j = 0; j < n_; ++j) sqrt_eig_[size_t(j)] = std::sqrt(std::max(lam_c[size_t(j)], 1e-20));
            for (int a = 0; a < n_; ++a)
                for (int b = 0; b < n_; ++b) {
                    double s1 = 0.0, s2 = 0.0;
                    for (int kk = 0; kk < n_; ++kk) {
                        double const p = v(a, kk) * v(b, kk);
                        s1 += p * sqrt_eig_[size_t(kk)];
                        s2 += p / sqrt_eig_[size_t(kk)];
                    }
                    sqrt_c_(a, b) = s1;
                    inv_sqrt_c_(a, b) = s2;
                }
        } // a failed decomposition keeps the previous one (dd_cmaes.cpp:346-351)
        acc_ = Mat(n_, 0.0);
    }
}

std::string DdCma::save() const {
    Writer w;
    header(w, CmaKind::DD, n_);
    w.pod<uint8_t>(active_ ? 1 : 0);
    w.pod<double>(sigma_);
    w.pod<double>(pc_factor_);
    w.pod<double>(pdc_factor_);
    w.pod<double>(ps_factor_);
    w.pod<uint64_t>(t_);
    for (vec const* v : {&mean_, &d_, &pc_, &pdc_, &ps_, &sqrt_eig_}) w.doubles(*v);
    for (Mat const* m : {&corr_, &sqrt_c_, &inv_sqrt_c_, &acc_}) w.doubles(m->a);
    w.text(rng_text(rng_, normal_));
    return w.out;
}

bool DdCma::restore(std::string const& blob, size_t pos) {
    Reader r{blob, pos};
    n_ = int(r.pod<uint32_t>());
    active_ = r.pod<uint8_t>() != 0;
    sigma_ = r.pod<double>();
    pc_factor_ = r.pod<double>();
    pdc_factor_ = r.pod<double>();
    ps_factor_ = r.pod<double>();
    t_ = r.pod<uint64_t>();
    for (vec* v : {&mean_, &d_, &pc_, &pdc_, &ps_, &sqrt_eig_}) *v = r.doubles();
    for (Mat* m : {&corr_, &sqrt_c_, &inv_sqrt_c_, &acc_}) {
        m->n = n_;
        m->a = r.doubles();
    }
    std::string const t = r.text();
    if (!r.ok || !rng_from_text(t, rng_, normal_)) return false;
    size_t const n = size_t(n_);
    for (vec* v : {&mean_, &d_, &pc_, &pdc_, &ps_, &sqrt_eig_})
        if (v->size() != n) return false;
    for (Mat* m : {&corr_, &sqrt_c_, &inv_sqrt_c_, &acc_})
        if (m->a.size() != n * n) return false;
    return true;
}

// ------------------------------------------------------------------ population / evolve

Population::Population(int size, vec const& lb, vec const& ub, uint32_t seed,
                       std::function<double(double const*)> const& fit) {
    std::mt19937 eng(seed);
    size_t const n = lb.size();
    for (int i = 0; i < size; ++i) {
        vec xi(n);
        for (size_t j = 0; j < n; ++j) xi[j] = std::uniform_real_distribution<double>(lb[j], ub[j])(eng);
        x.push_back(xi);
        f.push_back(0.0);
        set_xf(size_t(i), xi.data(), fit(xi.data()));
    }
}

void Population::set_xf(size_t i, double const* xi, double fi) {
    size_t const n = x[i].size();
    std::copy(xi, xi + n, x[i].begin());
    f[i] = fi;
    if (champion_x.empty() || less_f(fi, champion_f)) {
        champion_x.assign(xi, xi + n);
        champion_f = fi;
    }
}

size_t Population::best_idx() const {
    return size_t(std::min_element(f.begin(), f.end(), less_f) - f.begin());
}

size_t Population::worst_idx() const {
    return size_t(std::max_element(f.begin(), f.end(), less_f) - f.begin());
}

int evolve(Cma& cma, Population& pop, int gens, double ftol, double xtol,
           std::function<void(int, double const*, double*)> const& batch_fitness) {
    int const lam = int(pop.x.size());
    int const n = cma.dim();
    cma.new_evolve();
    std::vector<double> xs(size_t(lam) * n);
    vec fs(static_cast<size_t>(lam));
    for (int gen = 1; gen <= gens; ++gen) {
        cma.ask(lam, xs.data());
        double const best = pop.f[pop.best_idx()];
        double const df = std::fabs(best - pop.f[pop.worst_idx()]);
        if (cma.last_dx() < xtol || df < ftol) return gen - 1;
        batch_fitness(lam, xs.data(), fs.data());
        for (int i = 0; i < lam; ++i) pop.set_xf(size_t(i), &xs[size_t(i) * n], fs[size_t(i)]);
        cma.tell(lam, nullptr, fs.data());
    }
    return gens;
}

} // namespace ta3b::host
