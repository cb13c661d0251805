// Counters and the C entry that reads/resets them, for the operation-counting oracle build.
#include "opcount.hpp"
#undef double
thread_local OpCounts g_ops;
extern "C" void uwo_opcount(unsigned long long* out5, int reset)
{
    out5[0] = g_ops.add; out5[1] = g_ops.mul; out5[2] = g_ops.div; out5[3] = g_ops.sqrt; out5[4] = g_ops.tr;
    if (reset) g_ops = OpCounts{};
}
