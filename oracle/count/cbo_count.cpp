/* Counters of the operation-counting oracle build (see cbo_count.hpp). */
#include "cbo_count.hpp"
#undef double

extern "C" {
long long cbo_cnt[CNT_N];
void cbo_count_reset(void) { std::memset(cbo_cnt, 0, sizeof cbo_cnt); }
void cbo_count_read(long long *out) { std::memcpy(out, cbo_cnt, sizeof cbo_cnt); }
}
