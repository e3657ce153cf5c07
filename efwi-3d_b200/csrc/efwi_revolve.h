// Binomial checkpointing schedule of the exact-adjoint gradient (host code).
//
// The forward sweep produces states S_0 .. S_{nt-1} (S_0 = all zero).  The
// adjoint sweep runs blocks k = nt-1 .. 0 in that order, and block k needs
// S_k.  With s state slots in HBM (S_0 needs none) the blocks are reached by
// the recursive binomial schedule of Griewank (1992) and Griewank & Walther
// (2000, ACM TOMS 26, "Algorithm 799: revolve"), restated here:
//
//   rev(a, b, s): S_a is current and recoverable; run blocks b-1 .. a.
//     b - a == 1: block a.
//     s == 0:     for k = b-1 .. a: restore S_a, advance to S_k, block k.
//     otherwise:  t = least t with L(s, t) >= b - a, where
//                 L(s, t) = C(s + t + 1, t) is the longest chain that s slots
//                 reverse with each step advanced at most t times;
//                 d = min(l - 1, max(l - L(s-1, t), L(s, t-2), 1));
//                 advance to S_{a+d}, store it, rev(a+d, b, s-1),
//                 free the slot, restore S_a, rev(a, a+d, s).
//
// The split d is the smallest optimal one: the total number of forward
// steps is then t*l - C(s + t + 1, t - 1), the published minimum.  The
// first actions of the schedule are one uninterrupted sweep S_0 -> S_{nt-1},
// which is where the receivers are recorded, before the first block.
#pragma once
#include <cmath>
#include <vector>

namespace efwi {

enum CkOp { CK_ADVANCE = 0, CK_STORE = 1, CK_RESTORE = 2, CK_BLOCK = 3 };

struct CkAction {
  int op;
  int a;  // ADVANCE: from step a; STORE/RESTORE: slot (-1: the zero state S_0); BLOCK: k
  int b;  // ADVANCE: to step b (exclusive of the step that starts at b)
};

// C(s + t + 1, t), saturated at 1e18.
inline double ck_chain(int s, int t) {
  if (t < 0) return 0.0;
  double r = 1.0;
  for (int i = 1; i <= t; ++i) {
    r = r * (double)(s + 1 + i) / (double)i;
    if (r > 1e18) return 1e18;
  }
  return std::floor(r + 0.5);
}

struct CkPlan {
  std::vector<CkAction> actions;
  long long forward_steps = 0;
  int slots_used = 0;
  int repetitions = 0;  // t of the top level (1: every state stored)
  bool too_long = false;

  // Plans nt blocks with `slots` slots; gives up (too_long) when the
  // schedule would exceed max_actions actions.
  void build(int nt, int slots, long long max_actions) {
    actions.clear();
    forward_steps = 0;
    slots_used = 0;
    too_long = false;
    limit_ = max_actions;
    std::vector<int> free_slots;
    for (int k = slots - 1; k >= 0; --k) free_slots.push_back(k);
    free_ = &free_slots;
    total_slots_ = slots;
    repetitions = 0;
    if (nt < 1) return;
    if (nt > 1 && slots > 0) {
      int t = 1;
      while (ck_chain(slots, t) < nt) ++t;
      repetitions = t;
    } else if (nt > 1) {
      repetitions = nt - 1;
    }
    rev(0, nt, slots, -1);
  }

 private:
  long long limit_ = 0;
  std::vector<int> *free_ = nullptr;
  int total_slots_ = 0;

  void emit(int op, int a, int b) {
    if ((long long)actions.size() >= limit_) { too_long = true; return; }
    actions.push_back({op, a, b});
    if (op == CK_ADVANCE) forward_steps += b - a;
  }

  void rev(int a, int b, int s, int slot_a) {
    if (too_long) return;
    const int l = b - a;
    if (l == 1) { emit(CK_BLOCK, a, 0); return; }
    if (s == 0) {
      for (int k = b - 1; k >= a && !too_long; --k) {
        if (k != b - 1) emit(CK_RESTORE, slot_a, 0);
        if (k > a) emit(CK_ADVANCE, a, k);
        emit(CK_BLOCK, k, 0);
      }
      return;
    }
    int t = 1;
    while (ck_chain(s, t) < l) ++t;
    double d = std::max((double)l - ck_chain(s - 1, t), t >= 2 ? ck_chain(s, t - 2) : 1.0);
    d = std::max(d, 1.0);
    d = std::min(d, (double)(l - 1));
    const int m = a + (int)d;
    emit(CK_ADVANCE, a, m);
    const int slot = free_->back();
    free_->pop_back();
    const int used = total_slots_ - (int)free_->size();
    if (used > slots_used) slots_used = used;
    emit(CK_STORE, slot, 0);
    rev(m, b, s - 1, slot);
    free_->push_back(slot);
    emit(CK_RESTORE, slot_a, 0);
    rev(a, m, s, slot_a);
  }
};

}  // namespace efwi
