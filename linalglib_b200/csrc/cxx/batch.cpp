// Host-side planning of batched solves across GPUs.
#include "lab.h"

#include <algorithm>
#include <cstdint>
#include <vector>

namespace lab
{
    void set_error(const char* fmt, ...);
}

extern "C" {

// Size-balanced split of independent systems over nparts workers (GPUs): the
// largest system first, each to the worker with the least work so far (ties to
// the lower worker index; equal sizes keep their input order).  Host only.
LAB_API lab_status lab_batch_partition(int nsys, const int64_t* cost, int nparts, int* part)
{
    if(nsys < 0 || nparts <= 0 || (nsys > 0 && (!cost || !part)))
    {
        lab::set_error("lab_batch_partition: bad argument");
        return LAB_BAD_ARG;
    }
    std::vector<int> order((size_t)nsys);
    for(int k = 0; k < nsys; k++)
    {
        if(cost[k] < 0)
        {
            lab::set_error("lab_batch_partition: negative cost of system %d", k);
            return LAB_BAD_ARG;
        }
        order[(size_t)k] = k;
    }
    std::stable_sort(order.begin(), order.end(),
                     [&](int a, int b) { return cost[a] > cost[b]; });
    std::vector<int64_t> load((size_t)nparts, 0);
    for(int k : order)
    {
        int best = 0;
        for(int q = 1; q < nparts; q++)
            if(load[(size_t)q] < load[(size_t)best])
                best = q;
        part[k] = best;
        load[(size_t)best] += cost[k];
    }
    return LAB_OK;
}

} // extern "C"
