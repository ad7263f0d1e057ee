// Host-side verifiers of the AIR proof and of the a*b - c zerocheck proof (verifier.cu).
#pragma once
#include <array>
#include <cstddef>
#include <cstdint>
#include <vector>

#include "air_program.h"
#include "host.h"

namespace wl {

// Outcomes, valued as the C ABI's verifier statuses (AirVerifError, crates/air/src/verify.rs:26-34).
enum VerifyOutcome : int {
  VERIFY_OK = 0,
  VERIFY_PCS_COMMITMENT = 11,
  VERIFY_PCS_OPENING = 12,
  VERIFY_FS = 13,
  VERIFY_SUMCHECK = 14,
  VERIFY_SUM_MISMATCH = 16,
};

// A Merkle opening of a WHIR query, as offsets (in words) into proof_data: the opened row (128
// values), its authentication path (ll digests of 8 words, leaf level first) and the root it
// must reach; q is the leaf index.
struct MerkleOpening {
  uint64_t row, path, root;
  uint32_t q;
  int32_t ll;
};

// proof: proof_data as canonical u32 words; constants in Montgomery form.
// With log, the transcript as read (phases, challenges, queries, grinding witnesses) is recorded
// in the same form as the prover's (Transcript::log), up to the first failed check. The Merkle
// paths of each round's queries are checked on `threads` host threads (0: up to 16).
// With `defer`, the Merkle paths are not checked: every opening is appended to *defer (in
// transcript order) for a batched check, and the rest of the proof is checked as if they held.
// The verdict is then: if a listed opening fails, the proof is an opening error
// (VERIFY_PCS_OPENING), whatever the returned outcome, because every listed opening comes
// before the check that ended the replay; otherwise the returned outcome.
// With `prog`, the proof is of that constraint-program AIR (`air` is unused).
int verify_air_proof(const Settings& s, const AirConsts& air, const kb::P16Consts& p16, const kb::P24Consts& p24,
                     int log_n, const uint32_t* proof, size_t proof_len, TranscriptLog* log = nullptr,
                     int threads = 0, std::vector<MerkleOpening>* defer = nullptr,
                     const ProgramAir* prog = nullptr);
int verify_abc_proof(const kb::P16Consts& p16, int log_n, int skips, const uint32_t* proof, size_t proof_len);

}  // namespace wl
