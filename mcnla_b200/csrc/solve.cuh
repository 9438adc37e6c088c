// Whole solves of mcnla_b200_problem descriptors (stages.cu), shared by the
// server's workers (server.cu) and the grouped batch.
#pragma once
#include "common.cuh"

namespace mb {

// Device scratch a worker keeps across problems (grown stream-ordered on its
// context's stream): the FP64 copy of an FP32 A, and the BF16 parts of A and
// of A' when the problem does not bring its own.
struct SolveScratch {
  double* a64 = nullptr;
  size_t a64_bytes = 0;
  uint16_t* split = nullptr;
  size_t split_bytes = 0;
  uint16_t* tsplit = nullptr;
  size_t tsplit_bytes = 0;
};
void solve_scratch_free(Context* c, SolveScratch& s);
inline int64_t solve_scratch_bytes(const SolveScratch& s) {
  return int64_t(s.a64_bytes) + int64_t(s.split_bytes) + int64_t(s.tsplit_bytes);
}
// Scratch bytes a problem needs beyond its stage workspaces.
size_t problem_scratch_bytes(const mcnla_b200_problem& p);
// One whole solve (mcnla_b200_isvd, or mcnla_b200_isvd_mixed with the
// precision former) on the context's stream; fills p.iteration.
int solve_problem(Context* c, mcnla_b200_problem& p, SolveScratch& s);
// mcnla_b200_isvd_batched.
int batched_solve(int device, mcnla_b200_problem* problems, int count, int workers, int64_t budget);
// Host seconds of the last batch's phases (mcnla_b200_batched_times).
constexpr int kBatchPhases = 9;
int batched_times(double* seconds, int capacity);

}  // namespace mb
