// Test driver (CPU only): the bounded host wait of a compare launch
// (poll_with_limit) against fake stream queries: work that finishes, an
// error the stream reports, and a stall that never ends (injected on the
// host: the fake query answers "not ready" for good). No device is touched.
// Exit 0 when every check holds, else the number of the first failed check.
#include "dgpu_common.h"

#include <chrono>
#include <cstdio>

static int check(int no, bool ok) {
  if (!ok) std::printf("check %d failed\n", no);
  return ok ? 0 : no;
}

int main() {
  using namespace dgpu;
  int polls = 0;
  // finishes after 1000 polls
  cudaError_t e = poll_with_limit([&] { return ++polls < 1000 ? cudaErrorNotReady : cudaSuccess; }, 5.0);
  if (int r = check(1, e == cudaSuccess && polls == 1000)) return r;
  // an error reported by the stream passes through at once
  polls = 0;
  e = poll_with_limit([&] { return ++polls < 10 ? cudaErrorNotReady : cudaErrorIllegalAddress; }, 5.0);
  if (int r = check(2, e == cudaErrorIllegalAddress && polls == 10)) return r;
  // a stall: never ready; the wait gives up after the limit, not long after
  const auto t0 = std::chrono::steady_clock::now();
  e = poll_with_limit([] { return cudaErrorNotReady; }, 0.2);
  const double s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  if (int r = check(3, e == cudaErrorTimeout)) return r;
  if (int r = check(4, s >= 0.2 && s < 2.0)) return r;
  // the default limit, and the environment override read once
  if (int r = check(5, wait_limit_s() > 0.0)) return r;
  std::printf("ok\n");
  return 0;
}
