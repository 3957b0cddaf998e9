// The CUDA tracker's element maps compiled for the host (test infrastructure).
//
// bgt_kernel.cuh holds every per-particle map of the tracking kernel
// (decode, body_*, track1_rec and what they call) as __device__ functions
// with no other CUDA construct; with the qualifiers defined away a host C++
// compiler builds that same source.  The tables come from the same compiler
// bgt_create uses (bgt_compile.h), and the loop below is the warp-tile
// kernel's per-particle loop (track_kernel, TMODE 2): load the particle,
// clear the memos, the orbit_too_large check at the start, then turns x
// records with the loss element and turn recorded.
//
// Built with -ffp-contract=off (the device build's --fmad=false) the host
// build performs the same IEEE operations in the same order: double '/' and
// sqrt are correctly rounded on both sides, and every transcendental of a
// particle coordinate goes through bgt::cr, which is correctly rounded on
// both.  The tests check it bit for bit against the oracle -- the device
// source's arithmetic checked without a GPU -- and, built with
// -fsanitize=address, that no map reads outside its record.
#define __device__
#define __host__
#define __forceinline__ inline
#define __constant__

#include <math.h>
#include <stdint.h>
#include <stdio.h>

#include <string>
#include <vector>

#include "../bmad-ecosystem_b200/csrc/bgt_compile.h"
#include "../bmad-ecosystem_b200/csrc/bgt_kernel.cuh"

using namespace bgt;

namespace {

struct Tables {
  std::vector<double> all;
  std::vector<int64_t> off;
  int32_t table_dw = 0;
  bool rare = false;
};

template <bool RARE>
void track_one(Part& p, int32_t& ixe, int32_t& ixt, const double* table, const Glob& G, int32_t rec_begin,
               int32_t rec_end, int32_t turn0, int32_t n_turns) {
  const int32_t* seq = reinterpret_cast<const int32_t*>(table);
  DriftMemo memo;
  memo.pz = NAN;
  memo.a = 0;
  double qcol[QMEMO_CLASSES * 13];
  for (double& q : qcol) q = 0.0;
  const QMemo qmemo{qcol, 1};
  for (int c = 0; c < QMEMO_CLASSES; c++) qmemo.q[(c * 13 + 12) * qmemo.stride] = NAN;
  if (p.state == ALIVE && orbit_too_large(p, G)) {
    ixe = seq[2 * rec_begin + 1];
    ixt = turn0;
  }
  for (int t = 0; t < n_turns; t++) {
    if (p.state != ALIVE) break;
    const int turn = turn0 + t;
    for (int r = rec_begin; r < rec_end; r++) {
      if (p.state != ALIVE) break;
      track1_rec<RARE>(p, table + seq[2 * r], G, memo, qmemo);
      if (p.state != ALIVE) {
        ixe = seq[2 * r + 1];
        ixt = turn;
      }
    }
  }
}

}  // namespace

extern "C" {

// Track n particles (vec6 [6][n]) through records [rec_begin, rec_end) for
// n_turns turns, particle i in variant variant[i] (nullptr: variant 0).
// kernel: 0 the instance the host would pick (RARE when a record needs it),
// 1 the RARE instance always.  ix_turn_lost may be nullptr.  Returns 0,
// BGT_EINVAL or the table compiler's code with err filled.
int dmh_track(const bgt_element* eles, int32_t n_ele, int32_t n_variants, const bgt_species* sp,
              const int32_t* variant, double* vec6, double* beta, uint64_t* t, int32_t* state, int32_t* ix_ele_lost,
              int32_t* ix_turn_lost, int64_t n, int32_t rec_begin, int32_t rec_end, int32_t turn0,
              int32_t n_turns, int32_t kernel, char* err, int32_t err_len) {
  if (!eles || !sp || n_ele <= 0 || n_variants <= 0 || rec_begin < 0 || rec_end > n_ele || rec_begin > rec_end)
    return BGT_EINVAL;
  Tables T;
  std::string msg;
  int rc = host::compile_tables(eles, n_ele, n_variants, *sp, QMEMO_CLASSES, T.all, T.off, T.table_dw, T.rare,
                                msg);
  if (rc) {
    if (err && err_len > 0) snprintf(err, (size_t)err_len, "%s", msg.c_str());
    return rc;
  }
  host::c_multi_tables(c_cm, c_cm0);
  Glob G{};
  G.mc2 = sp->mass;
  G.mc2sq = sp->mass * sp->mass;
  G.p0c = eles[0].p0c;
  G.mal = sp->max_aperture_limit;
  G.ap_on = sp->aperture_limit_on;
  G.charge = sp->charge;
  G.abs_time = sp->absolute_time_tracking;
  G.abs_ref_shift = sp->absolute_time_ref_shift;
  G.track_time = t ? 1 : 0;
  // time tracking runs the RARE instances, as on the device
  const bool rare = T.rare || kernel == 1 || t != nullptr;
  for (int64_t i = 0; i < n; i++) {
    const int v = variant ? variant[i] : 0;
    if (v < 0 || v >= n_variants) return BGT_EINVAL;
    // each table alone in its own buffer, so that an address sanitizer sees
    // a read past the table's end
    std::vector<double> tab(T.all.begin() + T.off[v], T.all.begin() + T.off[v] + T.table_dw);
    Part p;
    p.x = vec6[0 * n + i];
    p.px = vec6[1 * n + i];
    p.y = vec6[2 * n + i];
    p.py = vec6[3 * n + i];
    p.z = vec6[4 * n + i];
    p.pz = vec6[5 * n + i];
    p.beta = beta[i];
    p.state = state[i];
    int32_t ixe = ix_ele_lost[i];
    int32_t ixt = ix_turn_lost ? ix_turn_lost[i] : -1;
    p.t_lo = t ? t[2 * i] : 0;
    p.t_hi = t ? t[2 * i + 1] : 0;
    if (rare)
      track_one<true>(p, ixe, ixt, tab.data(), G, rec_begin, rec_end, turn0, n_turns);
    else
      track_one<false>(p, ixe, ixt, tab.data(), G, rec_begin, rec_end, turn0, n_turns);
    vec6[0 * n + i] = p.x;
    vec6[1 * n + i] = p.px;
    vec6[2 * n + i] = p.y;
    vec6[3 * n + i] = p.py;
    vec6[4 * n + i] = p.z;
    vec6[5 * n + i] = p.pz;
    beta[i] = p.beta;
    state[i] = p.state;
    if (t) {
      t[2 * i] = p.t_lo;
      t[2 * i + 1] = p.t_hi;
    }
    ix_ele_lost[i] = ixe;
    if (ix_turn_lost) ix_turn_lost[i] = ixt;
  }
  return 0;
}

// Bytes of one variant's compiled table (what bgt_table_info reports), or a
// negative code when an element is rejected.
int64_t dmh_table_bytes(const bgt_element* eles, int32_t n_ele, int32_t n_variants, const bgt_species* sp) {
  Tables T;
  std::string msg;
  int rc = host::compile_tables(eles, n_ele, n_variants, *sp, QMEMO_CLASSES, T.all, T.off, T.table_dw, T.rare,
                                msg);
  return rc ? rc : (int64_t)T.table_dw * 8;
}

// Whether the compiled tables need the RARE kernel instance (1), do not (0),
// or a negative code when an element is rejected.
int dmh_needs_rare(const bgt_element* eles, int32_t n_ele, int32_t n_variants, const bgt_species* sp) {
  Tables T;
  std::string msg;
  int rc = host::compile_tables(eles, n_ele, n_variants, *sp, QMEMO_CLASSES, T.all, T.off, T.table_dw, T.rare,
                                msg);
  return rc ? rc : (T.rare ? 1 : 0);
}

}  // extern "C"
