// Specimen preparation on the host: slice assignment of atoms with erf weights, the Debye-Waller
// fold of Peng rows, and seeded frozen-phonon displacements, producing the coefficient rows the
// engine consumes (the inputs 3-8 of myProjectfun).
//
// Reference: CalAllEquilent20210223_lobato_peng.m:23-228 (slicing), CommonPart_forsimulation_
// lobato_peng.m:88-110 (Debye-Waller into Peng b), randshiftpos.m:1-44 (thermal displacements).
// Differences by design:
//  * the displacements come from a counter-based generator keyed by (seed, atom, draw, axis)
//    instead of MATLAB's rng('shuffle'): a configuration is reproducible from its seed and does
//    not depend on the order in which atoms are processed;
//  * an atom that cannot be placed inside the slab after kMaxDraws draws is an error instead of
//    an endless loop.
//
// Table layouts (getpotentialpara_lotabo_peng.m:26-84): the 16-column "nuclear" table
//   Z x y z B occ a1 b1 .. a5 b5
// and the 28-column "partly ionic" table
//   Z x y z B occ f_ion a1 b1 .. a5 b5 (ion) f_atom a1 b1 .. a5 b5 (atom).
#include <cmath>
#include <cstdint>
#include <limits>
#include <string>
#include <vector>

#include "common.cuh"

namespace {

constexpr int kNuclearCols = 16, kIonCols = 28;
constexpr int kMaxDraws = 100000;
const double kPi = 3.14159265358979323846;

int fail(int code, const char* msg) {
  totem::set_last_error(msg);
  return code;
}

// |erf(2 pi z2 / sqrt(b)) / 2 - erf(2 pi z1 / sqrt(b)) / 2|: the share of an atom's projected
// potential between z1 and z2 (CalAllEquilent20210223_lobato_peng.m:226)
double contribution(double b, double z1, double z2) {
  const double s = std::sqrt(b);
  return std::fabs(0.5 * std::erf(2.0 * kPi * z2 / s) - 0.5 * std::erf(2.0 * kPi * z1 / s));
}

struct SliceWindow {
  double lo, hi;       // atoms with lo <= z < hi take part in the slice
  double top, thick, reach;
  bool first, last;
  // z1 = z - (top + thick) and z2 = z - top, open-ended at the stack's ends and beyond reach
  void limits(double z, double* z1, double* z2) const {
    const double inf = std::numeric_limits<double>::infinity();
    *z1 = last ? -inf : z - (top + thick);
    *z2 = first ? inf : z - top;
    if (std::fabs(*z2) >= reach) *z2 = inf;
    if (std::fabs(*z1) >= reach) *z1 = -inf;
  }
};

SliceWindow window(const double* slicethick, int slices, int i, double eachthick, int multiceng) {
  SliceWindow w;
  w.top = slicethick[i];
  w.thick = eachthick;
  w.reach = multiceng * eachthick;
  w.lo = w.top - w.reach;
  w.hi = w.top + w.reach + eachthick;
  w.first = (i == 0);
  w.last = (i == slices - 1);
  return w;
}

// Atoms of every slice in table order, as offsets into one index list: slice i takes the atoms
// with lo(i) <= z < hi(i).  With the slice tops in increasing order (as ToTem writes them) each
// atom is placed by a binary search into the few slices its window reaches; otherwise every
// slice tests every atom.  The membership test is the same expression either way.
void slice_members(const double* t, int n, int ncol, const double* slicethick, int slices, double eachthick,
                   int multiceng, std::vector<long long>& beg, std::vector<int>& idx) {
  std::vector<SliceWindow> w(slices);
  bool sorted = true;
  for (int i = 0; i < slices; ++i) {
    w[i] = window(slicethick, slices, i, eachthick, multiceng);
    if (i && !(slicethick[i] > slicethick[i - 1])) sorted = false;
  }
  beg.assign(slices + 1, 0);
  auto each = [&](auto&& visit) {  // visit(slice, atom) in atom order
    for (int a = 0; a < n; ++a) {
      const double z = t[(size_t)a * ncol + 3];
      if (sorted) {
        int lo = 0, hi = slices;  // first slice whose window ends above z
        while (lo < hi) {
          const int mid = (lo + hi) / 2;
          if (w[mid].hi > z) hi = mid;
          else lo = mid + 1;
        }
        for (int i = lo; i < slices && w[i].lo <= z; ++i)
          if (z >= w[i].lo && z < w[i].hi) visit(i, a);
      } else {
        for (int i = 0; i < slices; ++i)
          if (z >= w[i].lo && z < w[i].hi) visit(i, a);
      }
    }
  };
  each([&](int i, int) { ++beg[i + 1]; });
  for (int i = 0; i < slices; ++i) beg[i + 1] += beg[i];
  idx.resize((size_t)beg[slices]);
  std::vector<long long> fill(beg.begin(), beg.end() - 1);
  each([&](int i, int a) { idx[(size_t)fill[i]++] = a; });
}

// Per-slice rows of one table: ``acols`` are the a_i columns scaled by the contribution with the
// b_i right after them; the row written drops Z, z and B (and appends B * dbmode for Lobato).
long long slice_table(const double* t, int n, int ncol, const std::vector<int>& acols, bool lobato, int dbmode,
                      const double* slicethick, int slices, double eachthick, int multiceng, double* out,
                      long long cap, double* series) {
  const int ocol = ncol - 3 + (lobato ? 1 : 0);
  std::vector<long long> beg;
  std::vector<int> idx;
  slice_members(t, n, ncol, slicethick, slices, eachthick, multiceng, beg, idx);
  std::vector<double> r(ncol);
  for (int i = 0; i < slices; ++i) {
    if (series) series[i] = (double)(beg[i + 1] - beg[i]);
    if (out == nullptr) continue;
    const SliceWindow w = window(slicethick, slices, i, eachthick, multiceng);
    for (long long q = beg[i]; q < beg[i + 1] && q < cap; ++q) {
      const double* src = t + (size_t)idx[(size_t)q] * ncol;
      for (int k = 0; k < ncol; ++k) r[k] = src[k];
      double z1, z2;
      w.limits(src[3], &z1, &z2);
      for (int c : acols) r[c] *= contribution(r[c + 1], z1, z2);
      double* dst = out + (size_t)q * ocol;
      int o = 0;
      for (int k = 0; k < ncol; ++k)
        if (k != 0 && k != 3 && k != 4) dst[o++] = r[k];
      if (lobato) dst[o++] = src[4] * dbmode;
    }
  }
  return beg[slices];
}

// SplitMix64 output function (Steele, Lea & Flood, "Fast splittable pseudorandom number
// generators", OOPSLA 2014), used here as a hash of the draw's key.
uint64_t mix64(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}

// Uniform in (0, 1] from 53 bits of the hash of (seed, atom, draw, axis, which).
double uniform(uint64_t seed, uint64_t atom, uint64_t draw, int axis, int which) {
  const uint64_t h = mix64(mix64(seed ^ mix64(atom)) ^ ((draw << 3) | (uint64_t)(axis * 2 + which)));
  return ((double)(h >> 11) + 1.0) * (1.0 / 9007199254740992.0);
}

// Standard normal by the Box-Muller transform of two uniforms.
double normal(uint64_t seed, uint64_t atom, uint64_t draw, int axis) {
  const double u1 = uniform(seed, atom, draw, axis, 0), u2 = uniform(seed, atom, draw, axis, 1);
  return std::sqrt(-2.0 * std::log(u1)) * std::cos(2.0 * kPi * u2);
}

}  // namespace

extern "C" {

int totem_slice_rows(int param, const double* nuclear, int n_nuclear, const double* nuc_ion, int n_ion,
                     double eachthick, const double* slicethick, int slices, int multiceng, int dbmode, double* ele_n,
                     long long cap_n, double* ele_n_i, long long cap_i, double* series_n, double* series_n_i,
                     long long* rows_n, long long* rows_i) {
  if (param != TOTEM_PARAM_PENG && param != TOTEM_PARAM_LOBATO) return fail(TOTEM_ERR_INVALID_ARG, "unknown param");
  if (n_nuclear < 0 || n_ion < 0 || slices < 0 || multiceng < 0 || !(eachthick > 0))
    return fail(TOTEM_ERR_INVALID_ARG, "sizes or slice thickness out of range");
  if ((n_nuclear > 0 && !nuclear) || (n_ion > 0 && !nuc_ion) || (slices > 0 && !slicethick) || !rows_n || !rows_i)
    return fail(TOTEM_ERR_INVALID_ARG, "NULL argument");
  const bool lobato = (param == TOTEM_PARAM_LOBATO);
  const std::vector<int> an = {6, 8, 10, 12, 14};
  const std::vector<int> ai = {7, 9, 11, 13, 15, 18, 20, 22, 24, 26};
  *rows_n = slice_table(nuclear, n_nuclear, kNuclearCols, an, lobato, dbmode, slicethick, slices, eachthick, multiceng,
                        ele_n, cap_n, series_n);
  *rows_i = slice_table(nuc_ion, n_ion, kIonCols, ai, lobato, dbmode, slicethick, slices, eachthick, multiceng,
                        ele_n_i, cap_i, series_n_i);
  if ((ele_n && *rows_n > cap_n) || (ele_n_i && *rows_i > cap_i))
    return fail(TOTEM_ERR_INVALID_ARG, "row buffers smaller than the rows produced (see rows_n / rows_i)");
  totem::set_last_error("");
  return TOTEM_OK;
}

int totem_fold_debye_waller(int param, double* nuclear, int n_nuclear, double* nuc_ion, int n_ion) {
  if (param != TOTEM_PARAM_PENG && param != TOTEM_PARAM_LOBATO) return fail(TOTEM_ERR_INVALID_ARG, "unknown param");
  if (n_nuclear < 0 || n_ion < 0 || (n_nuclear > 0 && !nuclear) || (n_ion > 0 && !nuc_ion))
    return fail(TOTEM_ERR_INVALID_ARG, "NULL argument or negative count");
  totem::set_last_error("");
  if (param == TOTEM_PARAM_LOBATO) return TOTEM_OK;  // Lobato rows keep B apart (exp(-B s^2))
  for (int a = 0; a < n_nuclear; ++a) {
    double* r = nuclear + (size_t)a * kNuclearCols;
    for (int c = 7; c < 16; c += 2) r[c] += r[4];
  }
  for (int a = 0; a < n_ion; ++a) {
    double* r = nuc_ion + (size_t)a * kIonCols;
    for (int c = 8; c < 17; c += 2) r[c] += r[4];
    for (int c = 19; c < 28; c += 2) r[c] += r[4];
  }
  return TOTEM_OK;
}

int totem_frozen_phonon(const double* table, int n, int ncol, double eachthick, const double* slicethick, int slices,
                        unsigned long long seed, double* out) {
  if (n < 0 || ncol < 5 || slices < 1 || !(eachthick > 0)) return fail(TOTEM_ERR_INVALID_ARG, "sizes out of range");
  if ((n > 0 && (!table || !out)) || !slicethick) return fail(TOTEM_ERR_INVALID_ARG, "NULL argument");
  const double lo = slicethick[0], hi = slicethick[slices - 1] + eachthick;
  for (int a = 0; a < n; ++a) {
    const double* src = table + (size_t)a * ncol;
    double* dst = out + (size_t)a * ncol;
    for (int k = 0; k < ncol; ++k) dst[k] = src[k];
    const double sig = std::sqrt(src[4] / 8.0 / kPi / kPi);
    int d = 0;
    for (;; ++d) {
      if (d == kMaxDraws) return fail(TOTEM_ERR_INVALID_ARG, "an atom could not be placed inside the slab");
      for (int k = 0; k < 3; ++k) dst[1 + k] = src[1 + k] + normal(seed, (uint64_t)a, (uint64_t)d, k) * sig;
      if (dst[3] >= lo && dst[3] < hi) break;
    }
  }
  totem::set_last_error("");
  return TOTEM_OK;
}

}  // extern "C"
