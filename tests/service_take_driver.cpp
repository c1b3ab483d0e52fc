// Test driver (CPU only): the denoising service's batching rule
// (dgpu_service::take) and length classes on hand-made requests. The
// service's device work is never started. Exit 0 when every check holds, else
// the number of the first failed check.
#include "dgpu_service.cpp"

#include <cstdio>

namespace dgpu {
void set_last_error(const char*) {}
int dada_batch_each(int, const dgpu_dada_params*, int, const uint32_t*, const char*, const uint32_t*,
                    const uint32_t*, const uint32_t*, const uint8_t*, const uint32_t*, const double*, int,
                    const std::function<void(size_t, dgpu_result*)>&) {
  return DGPU_E_UNSUPPORTED;
}
}  // namespace dgpu
extern "C" {
void dgpu_result_free(dgpu_result*) {}
const char* dgpu_last_error(void) { return ""; }
int dgpu_dada(int, const dgpu_dada_params*, int, const char*, const uint32_t*, const uint32_t*, const uint32_t*,
              const uint8_t*, const uint32_t*, const double*, int, dgpu_result**) {
  return DGPU_E_UNSUPPORTED;
}
}

static int check(int no, bool ok) {
  if (!ok) std::printf("check %d failed\n", no);
  return ok ? 0 : no;
}

int main() {
  int bad = 0;
  auto note = [&](int rc) {
    if (!bad) bad = rc;
  };
  note(check(1, length_class(200) == 0 && length_class(201) == 1 && length_class(600) == 1 &&
                    length_class(601) == 2));
  dgpu_service s;
  s.budget = 25;
  std::vector<Request> req(5);
  const int cls[5] = {0, 1, 0, 0, 2};
  const uint64_t fp[5] = {10, 10, 10, 10, 40};
  for (int i = 0; i < 5; ++i) {
    req[size_t(i)].id = uint64_t(i);
    req[size_t(i)].cls = cls[i];
    req[size_t(i)].footprint = fp[i];
  }
  std::vector<Request*> batch;
  uint64_t used = 0;
  note(check(2, !s.take(batch, used)));  // nothing pending
  for (int i = 0; i < 4; ++i) s.pending.push_back(&req[size_t(i)]);
  // the oldest request's class, in arrival order, while the budget holds
  note(check(3, s.take(batch, used) && batch.size() == 2 && batch[0]->id == 0 && batch[1]->id == 2 && used == 20 &&
                    s.in_flight == 20));
  note(check(4, s.pending.size() == 2 && s.pending[0]->id == 1 && s.pending[1]->id == 3));
  batch.clear();
  note(check(5, !s.take(batch, used) && batch.empty()));  // 20 in flight + 10 > 25
  s.in_flight -= 20;
  s.held = true;
  note(check(6, !s.take(batch, used)));  // held
  s.held = false;
  note(check(7, s.take(batch, used) && batch.size() == 1 && batch[0]->id == 1 && s.pending.size() == 1));
  s.in_flight -= used;
  batch.clear();
  // with nothing in flight the oldest request is taken even above the budget
  s.pending.push_front(&req[4]);
  note(check(8, s.take(batch, used) && batch.size() == 1 && batch[0]->id == 4 && used == 40 &&
                    s.pending.size() == 1 && s.pending[0]->id == 3));
  s.pending.clear();
  return bad;
}
