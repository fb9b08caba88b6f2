// ORACLE — test infrastructure only.
//
// A CPU restatement, in C++17, of the two-electron hot path of the Rust
// library nmrtist/integral (crate `integral`, version 0.4.3). It exists to
// check the CUDA product (integral_b200) and to time the reference algorithm
// on host cores. Only tests/, __graft_entry__.smoke() and bench.py's CPU
// baseline leg may load it; the product never links, imports or calls it.
//
// Every function restates the reference with the same operation order so that,
// compiled with -ffp-contract=off and without -ffast-math against glibc's libm
// (the libm Rust's f64::{exp,powf,cos,hypot} call on Linux), results are
// bit-for-bit those of the Rust code.  Rust's `powi` is lowered by LLVM to the
// square-and-multiply routine `__powidf2`, restated here as `powi`.
//
// Parity pins: Boys known values (crates/integral/src/math/boys.rs:468-520),
// the Rys moment identity (src/math/rys.rs:578-626), the Chebyshev Rys tables
// regenerated by the restated generator and compared against the literal
// coefficients of src/math/rys_tables.rs (fingerprint fixture in
// tests/golden), and the signed mpmath c2s tables of
// tests/c2s_independent_reference.rs.
#pragma once
#include <array>
#include <cstddef>
#include <cstdint>
#include <vector>

namespace oracle {

constexpr int MAX_L = 6;            // src/engine/os.rs:34
constexpr int MAX_GRAD_L = MAX_L - 1;  // src/grad.rs:50
constexpr int MAX_RYS_ROOTS = 13;   // src/math/rys.rs:104

using Vec3 = std::array<double, 3>;
using Tri = std::array<int, 3>;

// ---- L0: angular momentum / normalisation (src/math/am.rs, src/math/norm.rs)
inline int n_cart(int l) { return (l + 1) * (l + 2) / 2; }
std::vector<Tri> cart_components(int l);
int cart_index(const Tri& c);
double powi(double a, int b);
double double_factorial(long n);
double cart_norm(double alpha, int lx, int ly, int lz);

// ---- L0: Boys function (src/math/boys.rs)
double asymptotic_boundary(int m);
void boys_array(int m_max, double t, double* out);
void boys_reference(int m_max, double t, double* out);
const std::vector<double>& boys_table();  // 931 x 34 row-major

// ---- L0: Rys roots/weights (src/math/rys.rs + xtask/src/gen_rys_tables.rs)
constexpr int RYS_NC = 17;  // degree-16 Chebyshev series
void rys_roots_weights(int n, double t, double* roots, double* weights);
void rys_finite_reference(int n, double t, double* roots, double* weights);
// Generated Chebyshev tables: series [sub*n + i][k] for each n = 1..13.
struct RysTable {
  int n = 0;
  int n_sub = 0;
  double worst = 0.0;
  std::vector<double> root;    // n_sub*n*RYS_NC
  std::vector<double> weight;  // n_sub*n*RYS_NC
};
const std::vector<RysTable>& rys_tables();              // used at run time
const std::vector<RysTable>& rys_tables_regenerated();  // restated generator
bool rys_tables_are_reference_literals();

// ---- c2s (src/math/solid_harmonics.rs, src/spherical.rs)
std::vector<double> c2s_matrix(int l);
double monomial_to_raw_factor(int l);

// ---- basis (src/shell.rs)
struct Shell {
  int l = 0;
  bool spherical = false;
  Vec3 center{0, 0, 0};
  std::vector<double> exps;
  std::vector<double> coefs;
  int n_cart() const { return oracle::n_cart(l); }
  int n_func() const { return spherical ? 2 * l + 1 : oracle::n_cart(l); }
  int n_prim() const { return (int)exps.size(); }
  double primitive_coeff(int i) const;
};

enum class Engine { Auto = 0, OsHgp = 1, Rys = 2 };
Engine select_engine(int ne, int nf, int contraction_degree);

// Primitive-pair record (src/engine/os_eri.rs:188-198).
struct PrimPair {
  double zeta;
  Vec3 center;
  double kappa;
  double c1, c2;
  double inv_2zeta;
  Vec3 r1;
};
std::vector<PrimPair> build_pairs(const Shell& s1, const double* c1, const Shell& s2,
                                  const double* c2);

// OS/HGP shell quartet (src/engine/os_eri.rs:455-697, 2860-3143): accumulates
// the Cartesian block (row-major a,b,c,d) into `out`.
void os_shell_quartet(const Shell& a, const Shell& b, const Shell& c, const Shell& d,
                      const std::vector<PrimPair>& bra, const std::vector<PrimPair>& ket,
                      int la, int lb, int lc, int ld, double* out);
// Operator of the Rys primitive quartets below (process-wide, test use):
// 0 = Coulomb, > 0 = erf(omega r)/r (src/engine/rys.rs:101-172).  The OS/HGP
// engine has no attenuated path (as in the reference): erf callers use Rys.
void set_rys_erf_omega(double omega);
double rys_erf_omega();
// Rys primitive quartet (src/engine/rys.rs:121-231).
void rys_prim_quartet(double ea, const Vec3& A, int la, double eb, const Vec3& B, int lb,
                      double ec, const Vec3& C, int lc, double ed, const Vec3& D, int ld,
                      double scale, double* out);

class Basis {
 public:
  explicit Basis(std::vector<Shell> shells);
  const std::vector<Shell>& shells() const { return shells_; }
  int nsh() const { return (int)shells_.size(); }
  int nao() const { return nao_; }
  const std::vector<int>& offsets() const { return offs_; }
  const std::vector<Vec3>& atoms() const { return atoms_; }
  const std::vector<int>& shell_atom() const { return shell_atom_; }
  const std::vector<double>& eff(int s) const { return eff_[s]; }
  const std::vector<double>& c2s(int s) const { return c2s_[s]; }  // empty = Cartesian
  const std::vector<PrimPair>& pair_data(int i, int j) const;     // canonical i >= j

  // Function-space block of (ij|kl) with self-built pairs (eri_block_with).
  std::vector<double> eri_block(Engine e, int i, int j, int k, int l) const;
  // Function-space block with the canonical precomputed pair lists
  // (quartet_into_scratch_pairs); requires i >= j and k >= l.
  std::vector<double> eri_block_pairs(Engine e, int i, int j, int k, int l) const;
  std::vector<double> eri(Engine e) const;             // dense nao^4 (eri_with)
  std::vector<double> schwarz(Engine e) const;         // nsh^2 (schwarz_bounds_with)

 private:
  std::vector<Shell> shells_;
  int nao_ = 0;
  std::vector<int> offs_;
  std::vector<Vec3> atoms_;
  std::vector<int> shell_atom_;
  std::vector<std::vector<double>> eff_;
  std::vector<std::vector<double>> c2s_;
  std::vector<std::vector<PrimPair>> pair_data_;
};

// Cartesian -> function transform of a 4-index block (transform_block4_into).
std::vector<double> transform_block4(std::vector<double> block, const int dims[4],
                                     const std::vector<double>* mats[4]);

inline size_t tri_idx(size_t i, size_t j) { return i * (i + 1) / 2 + j; }

}  // namespace oracle
