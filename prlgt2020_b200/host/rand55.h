// The reference's noise generator on the host, so that the driver can run
// the same noise stream as the reference's own program: MyRand with
// __GEN_RAND55__ (a lagged-Fibonacci ring of 55 unsigned 64-bit words,
// MyRand.cc:73-110 and MyRand.h:81-91) and its Box-Muller normals of
// variance 1/2 (generate_gauss, MyRand.cc:115-130).  The draws per link are
// SU3rand's eight (MyMath.cc:256-292) in the reference's order: sites
// lexicographic, then mu (nspt.cc:365-423, one thread).
#pragma once

#include <cmath>
#include <cstdint>
#include <cstdio>

class Rand55 {
 public:
  explicit Rand55(long seed) {
    for (int i = 0; i < 54; i++) next_[i] = i + 1;
    next_[54] = 0;
    uint64_t tmp = (uint64_t)(161803398L + seed);  // Seed, MyRand.cc:30
    ring_[54] = tmp;
    uint64_t aux = 1;
    int j = 20;
    for (int i = 0; i < 54; i++, j += 21) {
      j %= 55;
      ring_[j] = aux;
      aux += tmp;
      tmp = ring_[j];
    }
    n1_ = 0;
    n2_ = 31;
    for (int k = 0; k < 55 * 4; k++) flat();
  }

  // uniform in [0, 1]: ring word / 2^64 (Norm_Factor = 1/ULONG_MAX, MyRand.h:44)
  double flat() {
    n1_ = next_[n1_];
    n2_ = next_[n2_];
    ring_[n1_] += ring_[n2_];
    return (double)ring_[n1_] * (1.0 / 18446744073709551616.0);
  }

  // normals of variance 1/2, in pairs (cos first, then the cached sin)
  double gauss() {
    if (!have_) {
      t_ = 6.28318530717959 * flat();  // MY_2pi, MyRand.h:40
      r_ = std::sqrt(-std::log(1. - flat()));
      have_ = true;
      return r_ * std::cos(t_);
    }
    have_ = false;
    return r_ * std::sin(t_);
  }

  void fill(double *out, long n) {
    for (long k = 0; k < n; k++) out[k] = gauss();
  }

  // The whole generator state as text (ring, links, positions, the cached
  // second normal of a Box-Muller pair), so that a resumed run draws the
  // numbers an uninterrupted one would.  Doubles go as hex floats: exact.
  void save(FILE *f) const {
    fprintf(f, "rand55 %d %d %d %a %a\n", n1_, n2_, have_ ? 1 : 0, r_, t_);
    for (int i = 0; i < 55; i++)
      fprintf(f, "%llu %d\n", (unsigned long long)ring_[i], next_[i]);
  }
  bool load(FILE *f) {
    int have = 0;
    if (fscanf(f, " rand55 %d %d %d %la %la", &n1_, &n2_, &have, &r_, &t_) != 5) return false;
    have_ = have != 0;
    for (int i = 0; i < 55; i++) {
      unsigned long long w = 0;
      if (fscanf(f, "%llu %d", &w, &next_[i]) != 2) return false;
      ring_[i] = (uint64_t)w;
    }
    return n1_ >= 0 && n1_ < 55 && n2_ >= 0 && n2_ < 55;
  }

 private:
  uint64_t ring_[55];
  int next_[55];
  int n1_, n2_;
  bool have_ = false;
  double r_ = 0.0, t_ = 0.0;
};
