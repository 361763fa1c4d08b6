// cj_tables.h -- host-side construction of the canonical Huffman tables
// (CJHuff) from a DHT segment's BITS/HUFFVAL lists.
#pragma once
#include <string.h>

#include "cj_core.h"

// Build `t` from the 16 code-length counts and their symbols (T.81 Annex C:
// codes are assigned in order of increasing length, each length continuing
// from the previous code shifted left by one).  The caller has already
// rejected over-subscribed lengths, so every code fits in its length.
inline void cj_build_huff(const uint8_t counts[16], const uint8_t* symbols, CJHuff* t) {
  memset(t->fast, 0, sizeof(t->fast));
  memset(t->vals, 0, sizeof(t->vals));
  int32_t code = 0;
  int k = 0;
  t->maxcode[0] = -1;
  t->valoff[0] = 0;
  for (int l = 1; l <= 16; l++) {
    int n = counts[l - 1];
    t->valoff[l] = k - code;
    for (int i = 0; i < n; i++, k++, code++) {
      uint8_t sym = symbols[k];
      t->vals[k & 255] = sym;
      if (l <= CJ_FAST_BITS) {
        int shift = CJ_FAST_BITS - l;
        uint16_t e = (uint16_t)((l << 8) | sym);
        for (int j = 0; j < (1 << shift); j++) t->fast[(code << shift) + j] = e;
      }
    }
    t->maxcode[l] = n ? code - 1 : -1;
    code <<= 1;
  }
  t->maxcode[17] = -1;
  t->valoff[17] = 0;
}

// Decode-step tables (CJSteps) of slot `slot` from its canonical table `t`
// (already built) and DHT counts; an undefined slot decodes nothing.
inline void cj_build_steps(const CJHuff& t, const uint8_t counts[16], bool defined, int slot, CJSteps* st) {
  const bool ac = slot >= 2;
  int pmin = 1 << CJ_FAST_BITS, pmax = -1;
  if (defined) cj_long_prefixes(counts, &pmin, &pmax);
  for (int p = 0; p < (1 << CJ_FAST_BITS); p++)
    st->pri[slot][p] = defined ? cj_step_primary(t, pmin, pmax, p, ac) : (uint16_t)CJ_STEP_BAD;
  for (int i = 0; i < CJ_STEP_SUBS; i++)
    for (int j = 0; j < 64; j++)
      st->sub[slot][i][j] = defined && pmin + i <= pmax ? cj_step_sub(t, pmin, i, j, ac) : (uint16_t)CJ_STEP_BAD;
}
