// Host-only check of the quantised four-wide records (traverse.cuh,
// quantize_record / q_decode): for random child boxes of many scales and
// offsets, every decoded box contains its exact box (outward rounding), and
// no decoded bound lies more than two steps outside it. Compiled with nvcc
// and run on the CPU by tests/test_quant_records.py; prints "ok <records>".
#include <cmath>
#include <cstdio>
#include <cstdint>
#include <cstring>
#include <random>

#include "../spatial_query_b200/csrc/traverse.cuh"

template <int D> int check(std::mt19937_64& rng, int records) {
  using QL = sq::QuantLayout<D>;
  std::uniform_real_distribution<double> u(0.0, 1.0);
  for (int r = 0; r < records; ++r) {
    const double scale = std::pow(10.0, -4.0 + 10.0 * u(rng));
    const double centre = (u(rng) - 0.5) * std::pow(10.0, -2.0 + 8.0 * u(rng));
    float box[8 * D];
    uint32_t codes[4];
    const int empty = int(u(rng) * 5.0) - 1;  // sometimes one empty slot
    for (int k = 0; k < 4; ++k) {
      codes[k] = (k == empty) ? sq::kNoHit : uint32_t(k + 1);
      for (int i = 0; i < D; ++i) {
        float a = float(centre + (u(rng) - 0.5) * scale);
        float b = (u(rng) < 0.1) ? a : float(centre + (u(rng) - 0.5) * scale);  // some flat boxes
        box[2 * D * k + i] = a < b ? a : b;
        box[2 * D * k + D + i] = a < b ? b : a;
      }
    }
    uint32_t out[QL::vec * 4];
    sq::quantize_record<D>(box, codes, out);
    for (int k = 0; k < 4; ++k) {
      if (out[QL::o_code + k] != codes[k]) { std::printf("code mismatch\n"); return 1; }
      if (codes[k] == sq::kNoHit) continue;
      for (int i = 0; i < D; ++i) {
        float o;
        std::memcpy(&o, &out[i], 4);
        const float step = sq::q_step(sq::q_byte(out + QL::o_exp, i));
        const uint32_t ql = sq::q_byte(out + QL::o_q, 2 * D * k + i), qh = sq::q_byte(out + QL::o_q, 2 * D * k + D + i);
        const float lo = sq::q_decode(o, ql, step), hi = sq::q_decode(o, qh, step);
        const float elo = box[2 * D * k + i], ehi = box[2 * D * k + D + i];
        if (!(lo <= elo && hi >= ehi)) {
          std::printf("not conservative: D=%d rec %d child %d axis %d: [%.9g, %.9g] vs exact [%.9g, %.9g]\n", D, r, k, i,
                      lo, hi, elo, ehi);
          return 1;
        }
        // tight: within two steps (plus the origin's rounding) of the exact bounds
        const double slack = 2.0 * double(step) + std::fabs(double(o)) * 1.2e-7;
        if (double(elo) - double(lo) > slack || double(hi) - double(ehi) > slack) {
          std::printf("loose: D=%d rec %d child %d axis %d: [%.9g, %.9g] vs exact [%.9g, %.9g], step %g\n", D, r, k, i,
                      lo, hi, elo, ehi, step);
          return 1;
        }
      }
    }
  }
  return 0;
}

int main() {
  std::mt19937_64 rng(12345);
  const int n = 20000;
  if (check<2>(rng, n) || check<3>(rng, n) || check<4>(rng, n) || check<6>(rng, n)) return 1;
  std::printf("ok %d\n", 4 * n);
  return 0;
}
