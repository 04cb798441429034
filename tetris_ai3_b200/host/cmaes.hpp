// Host-side CMA-ES for the island trainer: sep-CMA-ES and dd-CMA-ES restated
// from the reference's pagmo algorithms (ta3_trainer/src/pagmo/sep_cmaes.cpp,
// ta3_trainer/src/pagmo/dd_cmaes.cpp) as ask/tell optimisers, without Eigen or
// pagmo (neither is available): std::vector storage, a cyclic Jacobi
// eigensolver, std::mt19937 + std::normal_distribution sampling in the
// reference's draw order. Minimisation; NaN fitness ranks last.
//
// The reference runs `gens` generations inside one pagmo evolve() call and
// builds a fresh std::normal_distribution per call; new_evolve() marks that
// boundary (drops the distribution's cached deviate) so a trainer that calls
// it once per iteration draws the same normal stream as the reference.
#pragma once
#include <cstdint>
#include <functional>
#include <random>
#include <string>
#include <vector>

namespace ta3b::host {

using vec = std::vector<double>;

// strict weak order with NaN last (dd_cmaes.cpp:26-32, sep_cmaes.cpp:25-31)
inline bool less_f(double a, double b) {
    if (a != a) return false;
    if (b != b) return true;
    return a < b;
}

// dense row-major square matrix
struct Mat {
    int n = 0;
    vec a;
    Mat() = default;
    explicit Mat(int n_, double diag = 0.0) : n(n_), a(size_t(n_) * n_, 0.0) {
        for (int i = 0; i < n; ++i) a[size_t(i) * n + i] = diag;
    }
    double& operator()(int i, int j) { return a[size_t(i) * n + j]; }
    double operator()(int i, int j) const { return a[size_t(i) * n + j]; }
};

// Symmetric eigendecomposition by cyclic Jacobi rotations: A = V diag(w) V^T,
// eigenvector k in column k of V (V may be null for eigenvalues only).
// Returns false if the off-diagonal mass did not vanish within the sweep limit.
bool sym_eig(Mat const& A, vec& w, Mat* V);

enum class CmaKind : uint32_t { SEP = 1, DD = 2 };

class Cma {
public:
    virtual ~Cma() = default;
    virtual CmaKind kind() const = 0;
    int dim() const { return n_; }
    // the reference's per-evolve() boundary: a fresh normal distribution
    void new_evolve() { normal_ = std::normal_distribution<double>(0.0, 1.0); }
    // pagmo algorithm set_seed (dd_cmaes.cpp:361-364): re-seed the engine only
    void reseed(uint32_t seed) { rng_.seed(seed); }
    // Sample lam candidates, row-major into out (candidate i at out[i * dim]).
    virtual void ask(int lam, double* out) = 0;
    // Adapt from the fitness of k asked candidates: idx[j] is the candidate index
    // of fitness[j] (null idx: candidates 0..k-1). k == lam is the reference's
    // update; k < lam ranks and recombines only the evaluated subset.
    virtual void tell(int k, int const* idx, double const* fitness) = 0;
    // ||step|| of the last asked candidate (the reference's dx exit statistic)
    double last_dx() const { return last_dx_; }
    int asked() const { return asked_; }
    vec const& mean() const { return mean_; }
    virtual double sigma() const = 0;
    // per-axis standard deviation of the current search distribution
    virtual vec axis_std() const = 0;
    // k points (row-major) in the coordinates of the current search distribution: the map
    // under which it is N(0, I), i.e. the inverse of ask's x = m + sigma * A z
    virtual void whiten(int k, double const* x, double* z) const = 0;
    // Full adaptation state incl. the random engine and the normal
    // distribution's cached deviate: a restored optimiser continues identically.
    virtual std::string save() const = 0;
    static Cma* load(std::string const& blob, std::string* err = nullptr);

protected:
    int n_ = 0;
    vec mean_;
    double last_dx_ = 0.0;
    std::mt19937 rng_;
    std::normal_distribution<double> normal_{0.0, 1.0};
    int asked_ = 0;
    std::vector<double> z_;     // last asked N(0, I) draws, candidate-major (lam x n)
};

// sep_cmaes.cpp:66-279: diagonal covariance, c1 / cmu boosted by (n + 2) / 3.
class SepCma final : public Cma {
public:
    SepCma(vec const& x0, vec const& lb, vec const& ub, double sigma0, uint32_t seed);
    SepCma() = default;
    CmaKind kind() const override { return CmaKind::SEP; }
    void ask(int lam, double* out) override;
    void tell(int k, int const* idx, double const* fitness) override;
    double sigma() const override { return sigma_; }
    vec axis_std() const override;
    void whiten(int k, double const* x, double* z) const override;
    std::string save() const override;
    bool restore(std::string const& blob, size_t pos);

private:
    double sigma_ = 1.0;
    vec diag_, pc_, ps_, axis_;      // axis_: sqrt(diag) at the last ask
    std::vector<double> x_;          // last asked candidates (lam x n)
    uint64_t count_eval_ = 0;
};

// dd_cmaes.cpp:62-358: diagonal decoding D (fast, sep-like rate) times a
// correlation matrix C (slow, full rate), active negative-weight update,
// C and C^(+-1/2) refreshed from the accumulated update every teig generations.
class DdCma final : public Cma {
public:
    DdCma(vec const& x0, vec const& lb, vec const& ub, double sigma0, uint32_t seed, bool active = true);
    DdCma() = default;
    CmaKind kind() const override { return CmaKind::DD; }
    void ask(int lam, double* out) override;
    void tell(int k, int const* idx, double const* fitness) override;
    double sigma() const override { return sigma_; }
    vec axis_std() const override;
    void whiten(int k, double const* x, double* z) const override;
    std::string save() const override;
    bool restore(std::string const& blob, size_t pos);

private:
    bool active_ = true;
    double sigma_ = 1.0, pc_factor_ = 0.0, pdc_factor_ = 0.0, ps_factor_ = 0.0;
    vec d_, pc_, pdc_, ps_, sqrt_eig_;
    Mat corr_, sqrt_c_, inv_sqrt_c_, acc_;
    std::vector<double> y_;          // sqrtC z of the last ask (lam x n)
    uint64_t t_ = 0;
};

// ---- a pagmo-like population and evolve() for the optimiser's own tests

struct Population {
    std::vector<vec> x;
    vec f;
    vec champion_x;
    double champion_f = 0.0 / 0.0;
    // pagmo::population{prob, size, seed}: uniform in the box from mt19937(seed), each evaluated
    Population(int size, vec const& lb, vec const& ub, uint32_t seed, std::function<double(double const*)> const& fit);
    void set_xf(size_t i, double const* xi, double fi);
    size_t best_idx() const;
    size_t worst_idx() const;
};

// One reference evolve() call: `gens` generations of ask / evaluate / tell
// with the dx < xtol and |best - worst| < ftol exits checked on the previous
// generation (dd_cmaes.cpp:203-354, sep_cmaes.cpp:168-274). Returns the
// generations completed.
int evolve(Cma& cma, Population& pop, int gens, double ftol, double xtol,
           std::function<void(int lam, double const* xs, double* fs)> const& batch_fitness);

} // namespace ta3b::host
