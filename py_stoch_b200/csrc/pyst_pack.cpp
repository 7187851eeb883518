// Host-side packing of a model description into the device blob.
//
// Replaces the reference's per-model data preparation: the sparse char4
// lists of Parser.flatten_matrix (mod/parser/parser.py:58-71), the HOR
// vectors of TlParser.get_hors (mod/parser/tl_parser.py:98-120) and the
// __constant__ uploads (mod/simulator/cuTauLeaping/cuTauLeaping.py:86-107).
// The blob has no int8/uint8 limits: 16-bit indices, 16-bit stoichiometry.
#include <math.h>
#include <stdint.h>
#include <string.h>

#include <vector>

#include "pystoch_b200.h"

namespace {

uint32_t f32_bits(float f) {
  uint32_t u;
  memcpy(&u, &f, 4);
  return u;
}

struct Packed {
  std::vector<uint32_t> w;
};

int pack(const pyst_model_desc* m, Packed* out) {
  if (!m) return PYST_EINVAL;
  const int S = m->n_species, R = m->n_reactions;
  if (S < 1 || R < 1) return PYST_EINVAL;
  if (S > PYST_MAX_SPECIES || R > PYST_MAX_REACTIONS) return PYST_EUNSUPPORTED;
  if (!m->order || !m->pre || !m->net_change || !m->rate || !m->x0 ||
      !m->sample_times || !m->out_species)
    return PYST_EINVAL;
  if (m->n_samples < 1 || m->n_out < 1) return PYST_EINVAL;
  if (m->n_samples > (1 << 24) || m->n_out > S) return PYST_EUNSUPPORTED;
  if (!(m->eta > 0.0f) || m->n_c < 0) return PYST_EINVAL;
  for (int f = 0; f < m->n_samples; ++f) {
    const float t = m->sample_times[f];
    if (!isfinite(t) || t < 0.0f) return PYST_EINVAL;
    if (f > 0 && t < m->sample_times[f - 1]) return PYST_EINVAL;
  }
  for (int k = 0; k < m->n_out; ++k)
    if (m->out_species[k] < 0 || m->out_species[k] >= S) return PYST_EINVAL;
  for (int i = 0; i < S; ++i)
    if (m->x0[i] < 0) return PYST_EINVAL;
  for (int j = 0; j < R; ++j) {
    const float r = (float)m->rate[j];
    if (!isfinite(r) || r < 0.0f) return PYST_EINVAL;
  }
  auto idx = [&](int i, int j) { return (size_t)i * R + j; };
  for (int i = 0; i < S; ++i)
    for (int j = 0; j < R; ++j) {
      const int o = m->order[idx(i, j)];
      const int v = m->net_change[idx(i, j)];
      if (o < 0 || o > 255) return PYST_EUNSUPPORTED;
      if (v < -32767 || v > 32767) return PYST_EUNSUPPORTED;
      if (m->pre[idx(i, j)] < 0) return PYST_EINVAL;
    }

  std::vector<uint32_t>& w = out->w;
  w.assign(PYST_H_WORDS_HEADER, 0u);
  auto here = [&]() { return (uint32_t)w.size(); };

  w[PYST_H_OFF_RATE] = here();
  for (int j = 0; j < R; ++j) w.push_back(f32_bits((float)m->rate[j]));

  // reactant factors, reaction-major, species ascending
  std::vector<uint32_t> ptr, ent;
  ptr.push_back(0);
  for (int j = 0; j < R; ++j) {
    for (int i = 0; i < S; ++i) {
      const int o = m->order[idx(i, j)];
      if (o > 0) {
        const uint32_t fall = m->falling ? (m->falling[idx(i, j)] ? 1u : 0u)
                                         : 1u;
        ent.push_back((uint32_t)i | ((uint32_t)o << 16) | (fall << 24));
      }
    }
    ptr.push_back((uint32_t)ent.size());
  }
  w[PYST_H_NFAC] = (uint32_t)ent.size();
  w[PYST_H_OFF_FACPTR] = here();
  w.insert(w.end(), ptr.begin(), ptr.end());
  w[PYST_H_OFF_FAC] = here();
  w.insert(w.end(), ent.begin(), ent.end());

  // net change, reaction-major
  ptr.assign(1, 0);
  ent.clear();
  for (int j = 0; j < R; ++j) {
    for (int i = 0; i < S; ++i) {
      const int v = m->net_change[idx(i, j)];
      if (v != 0)
        ent.push_back((uint32_t)i | ((uint32_t)(uint16_t)(int16_t)v << 16));
    }
    ptr.push_back((uint32_t)ent.size());
  }
  w[PYST_H_NNET] = (uint32_t)ent.size();
  w[PYST_H_OFF_NETPTR] = here();
  w.insert(w.end(), ptr.begin(), ptr.end());
  w[PYST_H_OFF_NET] = here();
  w.insert(w.end(), ent.begin(), ent.end());

  w[PYST_H_OFF_TIMES] = here();
  for (int f = 0; f < m->n_samples; ++f) w.push_back(f32_bits(m->sample_times[f]));
  w[PYST_H_OFF_OUT] = here();
  for (int k = 0; k < m->n_out; ++k) w.push_back((uint32_t)m->out_species[k]);
  w[PYST_H_OFF_X0] = here();
  for (int i = 0; i < S; ++i) w.push_back((uint32_t)m->x0[i]);

  // net change, species-major (every species)
  ptr.assign(1, 0);
  ent.clear();
  for (int i = 0; i < S; ++i) {
    for (int j = 0; j < R; ++j) {
      const int v = m->net_change[idx(i, j)];
      if (v != 0)
        ent.push_back((uint32_t)j | ((uint32_t)(uint16_t)(int16_t)v << 16));
    }
    ptr.push_back((uint32_t)ent.size());
  }
  w[PYST_H_NSPV] = (uint32_t)ent.size();
  w[PYST_H_OFF_SPVPTR] = here();
  w.insert(w.end(), ptr.begin(), ptr.end());
  w[PYST_H_OFF_SPV] = here();
  w.insert(w.end(), ent.begin(), ent.end());

  // tau-selection word per species: H | H_type << 8 | reactant << 16
  w[PYST_H_OFF_G] = here();
  for (int i = 0; i < S; ++i) {
    int reactant = 0;
    for (int j = 0; j < R; ++j)
      if (m->pre[idx(i, j)] > 0) reactant = 1;
    const int H = m->hor ? m->hor[i] : 0;
    const int Ht = m->hor_type ? m->hor_type[i] : 0;
    if (H < 0 || H > 255 || Ht < 0 || Ht > 255) return PYST_EINVAL;
    w.push_back((uint32_t)H | ((uint32_t)Ht << 8) | ((uint32_t)reactant << 16));
  }

  // negative net-change entries per reaction (critical-reaction test)
  ptr.assign(1, 0);
  ent.clear();
  for (int j = 0; j < R; ++j) {
    for (int i = 0; i < S; ++i) {
      const int v = m->net_change[idx(i, j)];
      if (v < 0) ent.push_back((uint32_t)i | ((uint32_t)(-v) << 16));
    }
    ptr.push_back((uint32_t)ent.size());
  }
  w[PYST_H_NCRIT] = (uint32_t)ent.size();
  w[PYST_H_OFF_CRITPTR] = here();
  w.insert(w.end(), ptr.begin(), ptr.end());
  w[PYST_H_OFF_CRIT] = here();
  w.insert(w.end(), ent.begin(), ent.end());

  // general kinetic laws: program ranges, words, FP64 constants
  uint32_t nlaw = 0;
  if (m->law_ptr) {
    if (m->law_ptr[0] != 0) return PYST_EINVAL;
    for (int j = 0; j < R; ++j) {
      if (m->law_ptr[j + 1] < m->law_ptr[j]) return PYST_EINVAL;
      if (m->law_ptr[j + 1] > m->law_ptr[j]) ++nlaw;
    }
    const int ncode = m->law_ptr[R];
    if (ncode > 0 && !m->law_code) return PYST_EINVAL;
    if (m->n_law_const < 0 || (m->n_law_const > 0 && !m->law_const))
      return PYST_EINVAL;
    // check every program: known op codes, operands in range, and a
    // stack that never underflows, never exceeds 8 and ends at 1
    for (int j = 0; j < R; ++j) {
      if (m->law_ptr[j + 1] == m->law_ptr[j]) continue;
      int depth = 0;
      for (int c = m->law_ptr[j]; c < m->law_ptr[j + 1]; ++c) {
        const uint32_t op = m->law_code[c] >> 24, arg = m->law_code[c] & 0xFFFFFFu;
        int pops = 0, pushes = 1;
        if (op == 1) {
          if ((int)arg >= S) return PYST_EINVAL;
        } else if (op == 2) {
          if ((int)arg >= m->n_law_const) return PYST_EINVAL;
        } else if (op >= 3 && op <= 7) {
          pops = 2;
        } else if (op == 8 || (op >= 10 && op <= 15)) {
          pops = 1;
        } else if (op == 16) {
          pops = 1;
          pushes = 2;
        } else {
          return PYST_EINVAL;
        }
        if (depth < pops) return PYST_EINVAL;
        depth += pushes - pops;
        if (depth > 8) return PYST_EUNSUPPORTED;
      }
      if (depth != 1) return PYST_EINVAL;
    }
    w[PYST_H_OFF_LAWPTR] = here();
    for (int j = 0; j <= R; ++j) w.push_back((uint32_t)m->law_ptr[j]);
    w[PYST_H_OFF_LAW] = here();
    for (int c = 0; c < ncode; ++c) w.push_back(m->law_code[c]);
    if (w.size() & 1) w.push_back(0u);
    w[PYST_H_OFF_LAWC] = here();
    for (int k = 0; k < m->n_law_const; ++k) {
      uint64_t b;
      memcpy(&b, &m->law_const[k], 8);
      w.push_back((uint32_t)b);
      w.push_back((uint32_t)(b >> 32));
    }
  }

  while (w.size() & 3) w.push_back(0u);
  if (w.size() > (size_t)PYST_MAX_BLOB_WORDS) return PYST_EUNSUPPORTED;

  w[PYST_H_MAGIC] = PYST_BLOB_MAGIC;
  w[PYST_H_WORDS] = (uint32_t)w.size();
  w[PYST_H_S] = (uint32_t)S;
  w[PYST_H_R] = (uint32_t)R;
  w[PYST_H_KAPPA] = (uint32_t)m->n_out;
  w[PYST_H_ITA] = (uint32_t)m->n_samples;
  w[PYST_H_NC] = (uint32_t)m->n_c;
  w[PYST_H_ETA] = f32_bits(m->eta);
  w[PYST_H_FLAGS] = 0;
  w[PYST_H_NLAW] = nlaw;
  uint64_t tb;
  memcpy(&tb, &m->t_max, 8);
  w[PYST_H_TMAX_LO] = (uint32_t)tb;
  w[PYST_H_TMAX_HI] = (uint32_t)(tb >> 32);
  return PYST_OK;
}

}  // namespace

extern "C" {

int pyst_model_blob_words(const pyst_model_desc* model, int64_t* n_words) {
  if (!n_words) return PYST_EINVAL;
  Packed p;
  const int rc = pack(model, &p);
  if (rc) return rc;
  *n_words = (int64_t)p.w.size();
  return PYST_OK;
}

int pyst_model_build(const pyst_model_desc* model, uint32_t* blob,
                     int64_t n_words) {
  if (!blob) return PYST_EINVAL;
  Packed p;
  const int rc = pack(model, &p);
  if (rc) return rc;
  if ((int64_t)p.w.size() > n_words) return PYST_EINVAL;
  memcpy(blob, p.w.data(), p.w.size() * 4);
  return PYST_OK;
}

}  // extern "C"
