// Launch-shape autotuning cache (kq_tune.cu).
//
// Tuned shapes are stored one per line, "<gpu name>|<key> <values...>", in the file named by KUQCD_TUNE_CACHE, or
// $HOME/.cache/kuqcd_b200/tunecache.txt.  A missing or unwritable file only disables the cache.
#pragma once
#include <string>

namespace kq {

struct BatchTune {
    int bs;           // threads per CTA
    int ctas_per_sm;  // resident CTAs per SM of the persistent grid
    int rhs;          // right-hand sides per CTA: systems on one gauge field that share each link load (1,2,4,8)
    int spt;          // sites per thread: a tile is spt x bs sites
    int p64;          // right-hand sides per pass of the FP64 dslash (1, 2, 4): link reuse against occupancy
};

bool tune_lookup(const std::string &key, BatchTune *out);
void tune_store(const std::string &key, const BatchTune &t);

// single-system dslash block size (threads per CTA), keyed by lattice and precision pair
bool tune_lookup_int(const std::string &key, int *out);
void tune_store_int(const std::string &key, int v);

}  // namespace kq
