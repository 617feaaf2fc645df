// Owner-computes partition of a batch with overlapping outputs over several
// GPUs (host code only; no reference counterpart -- the reference runs one
// device).
//
// In the xbatched and pbatched layouts several entries may add into one
// output column (Ylist[k] == Ylist[k'], the aliasing contract of
// kronmult6_pbatched.hpp:52-66 and kronmult_xbatched.hpp:17-162).  Cutting
// such a batch across GPUs at arbitrary entries would leave partial sums of
// one output on several GPUs, to be reduced afterwards.  Here every output
// index goes to exactly one rank, together with every entry that adds into
// it, so each rank's kernels finish its outputs alone and no reduction
// crosses NVLink:
//   - the entries are sorted by output index (stable: entries of one output
//     keep their order, the order of the deterministic segmented mode);
//   - rank r takes one contiguous range of output indices,
//     [out_bounds[r], out_bounds[r+1]), and the entries that write them,
//     entry_order[entry_bounds[r] .. entry_bounds[r+1]);
//   - cut r is the start of the output group nearest to r B / R entries
//     (B entries, R ranks), never before cut r-1, so the entry counts are as
//     even as the output groups allow (entries of one shape cost the same).
// out_bounds[0] = 0 and out_bounds[R] = 1 + the largest output index.
#include <algorithm>
#include <new>
#include <numeric>
#include <vector>

#include "kronmult.h"

extern "C" int kron_owner_partition(int batchCount, int const ylist[], int nranks,
                                    int entry_order[], int entry_bounds[], int out_bounds[])
{
  if (batchCount < 0 || nranks < 1 || !entry_bounds || !out_bounds)
    return KRON_ERROR_INVALID_VALUE;
  if (batchCount > 0 && (!ylist || !entry_order))
    return KRON_ERROR_INVALID_VALUE;
  for (int k = 0; k < batchCount; k++)
    if (ylist[k] < 0)
      return KRON_ERROR_INVALID_VALUE;
  if (batchCount == 0)
  {
    for (int r = 0; r <= nranks; r++)
    {
      entry_bounds[r] = 0;
      out_bounds[r]   = 0;
    }
    return KRON_SUCCESS;
  }
  try
  {
    std::vector<int> order(batchCount);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(),
                     [&](int a, int b) { return ylist[a] < ylist[b]; });
    // positions where an output group starts, and the end of the batch
    std::vector<int> starts;
    starts.reserve(batchCount + 1);
    for (int p = 0; p < batchCount; p++)
      if (p == 0 || ylist[order[p]] != ylist[order[p - 1]])
        starts.push_back(p);
    starts.push_back(batchCount);

    const int ymax = ylist[order[batchCount - 1]];
    entry_bounds[0] = 0;
    out_bounds[0]   = 0;
    int prev        = 0;
    for (int r = 1; r < nranks; r++)
    {
      const long long target = (long long)batchCount * r / nranks;
      // nearest group start to the target, not before the previous cut
      auto it = std::lower_bound(starts.begin(), starts.end(), (int)target);
      int cut = (it == starts.end()) ? batchCount : *it;
      if (it != starts.begin())
      {
        const int below = *(it - 1);
        if (target - below < (long long)cut - target)
          cut = below;
      }
      cut             = std::max(cut, prev);
      entry_bounds[r] = cut;
      out_bounds[r]   = cut < batchCount ? ylist[order[cut]] : ymax + 1;
      prev            = cut;
    }
    entry_bounds[nranks] = batchCount;
    out_bounds[nranks]   = ymax + 1;
    std::copy(order.begin(), order.end(), entry_order);
  }
  catch (const std::bad_alloc &)
  {
    return KRON_ERROR_ALLOC;
  }
  return KRON_SUCCESS;
}
