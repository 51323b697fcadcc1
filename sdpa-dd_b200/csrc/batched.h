// Batched Newton core of the batch solver (batched.cu): the Schur build
// and Cholesky of B of many problems at once, as one captured CUDA graph of
// persistent launches, bit for bit the single-problem results.
#pragma once

#include <condition_variable>
#include <mutex>
#include <string>

#include "context.h"

namespace sddd {

// True when c's problem can take the batched core: one SDP block whose
// constraints are all dense F1/F2 owners, m <= 1024, n <= 128, plain form.
bool core_eligible(const Context &c);

class CoreEngine {
  public:
    explicit CoreEngine(int device);
    ~CoreEngine();
    CoreEngine(const CoreEngine &) = delete;
    CoreEngine &operator=(const CoreEngine &) = delete;
    // A worker starts / ends a solve (the engine waits for at most the
    // active workers before it launches).
    void enter();
    void leave();
    // Schur build and Cholesky of B of c (eligible), batched with the other
    // workers' problems; returns LAPACK's info.
    int schur_factor(Context &c);
    // The autotuner's tile shape per size class of m.
    std::string tuning() const;

  private:
    struct Impl;
    Impl *p = nullptr;
    std::mutex mu;
    std::condition_variable cv;
    int active = 0;
    unsigned long generation = 0;
    // a gathering whose launch failed: its members report the error
    unsigned long failed_generation = ~0ul;
    std::string failed_msg;
    void launch_locked();
    void launch_or_fail_locked();
};

} // namespace sddd
