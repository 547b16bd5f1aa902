// Host-side harness for the bit-sliced circuit header (test infrastructure).
// Compiles the same __host__ __device__ code the CUDA kernels run and exposes
// it to pytest so the circuit can be compared with the oracle without a GPU.
#include <stdint.h>
#include "../../iris-mpc_b200/csrc/circuit.cuh"

using namespace irs;

extern "C" int harness_threshold_words(const uint16_t* const* code, const uint16_t* const* mask, long n_words,
                                       uint32_t threshold_a, const uint32_t* keys, uint32_t dev, uint64_t batch,
                                       uint64_t word_base, int stage, uint32_t* revealed, uint32_t* msb_comp) {
  for (long w = 0; w < n_words; w++) {
    WordRand wr;
    for (int s = 0; s < 3; s++)
      for (int i = 0; i < 8; i++) wr.key[s].k[i] = keys[8 * s + i];
    wr.nonce = nonce_of(kDomCircuit, dev);
    wr.base = counter_of(batch, (word_base + (uint64_t)w) * kCircuitBlocksPerWord);
    const uint16_t* c[3] = {code[0] + 32 * w, code[1] + 32 * w, code[2] + 32 * w};
    const uint16_t* m[3] = {mask[0] + 32 * w, mask[1] + 32 * w, mask[2] + 32 * w};
    Comp msb;
    uint32_t r = stage == kStageFull ? threshold_word<kStageFull>(c, m, threshold_a, wr, msb)
                                     : threshold_word<kStageMsbOnly>(c, m, threshold_a, wr, msb);
    revealed[w] = r;
    msb_comp[0 * n_words + w] = msb.c0;
    msb_comp[1 * n_words + w] = msb.c1;
    msb_comp[2 * n_words + w] = msb.c2;
  }
  return 0;
}

extern "C" void harness_chacha_block(const uint32_t* key, uint64_t counter, uint64_t nonce, int rounds,
                                     uint32_t* out) {
  ChaChaKey k;
  for (int i = 0; i < 8; i++) k.k[i] = key[i];
  if (rounds == 20) chacha_block<20>(k, counter, nonce, out);
  else chacha_block<12>(k, counter, nonce, out);
}

extern "C" void harness_packed16(const uint32_t* a, const uint32_t* b, uint32_t* add, uint32_t* sub, long n) {
  for (long i = 0; i < n; i++) {
    add[i] = add2(a[i], b[i]);
    sub[i] = sub2(a[i], b[i]);
  }
}

extern "C" void harness_slice16(const uint32_t* w, uint32_t* planes) { slice16(w, planes); }

extern "C" void harness_transpose32(uint32_t* a) { transpose32(a); }
