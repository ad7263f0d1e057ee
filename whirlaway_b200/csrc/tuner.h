// Autotuner of kernel launch plans. Several kernels of the commitment have launch plans that
// compute the same result with different shapes: the LDE's split of its stages into passes and
// the persistent passes' blocks per SM, the leaf sponges' rows per block, and the width from
// which a Merkle level runs one compression per thread; and the inner sums' staging of the
// witness (cp.async per thread, or bulk copies by the TMA engine on an mbarrier pipeline).
// Which plan is fastest depends on the
// table's shape (rows, columns, element size). The first time a tuning context meets a shape it
// runs every plan on the real data (each writes the same output), times them with CUDA events
// and keeps the fastest for that device and shape; later proofs of the shape, on any context
// or server worker, use the kept plan.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace wl {

enum TuneFamily { TUNE_LDE = 0, TUNE_LEAF = 1, TUNE_MERKLE = 2, TUNE_INNER = 3, TUNE_FAMILIES = 4 };

const char* tune_family_name(int family);
int tune_plan_count(int family);
int tune_default_plan(int family);
// Family by name ("lde", "leaf", "merkle", "inner"), -1 if unknown.
int tune_family_from_name(const char* name);
// A plan forced for every shape of a family (-1: none), process-wide; for tests and sweeps.
void tune_force(int family, int plan);
int tune_forced(int family);
// The kept plan for (device, family, shape key), -1 when the shape has not been tuned.
int tune_lookup(int device, int family, uint64_t key);
void tune_store(int device, int family, uint64_t key, int plan, const std::vector<float>& ms);
// Forgets every kept plan.
void tune_clear();
// {"lde": [{"device": d, "key": k, "plan": p, "ms": [...]}, ...], ...}
std::string tune_json();

}  // namespace wl
