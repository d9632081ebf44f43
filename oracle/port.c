/*
 * port.c — CPU restatement of the reference hot path, in plain C.
 *
 * TEST INFRASTRUCTURE ONLY (the oracle).  Loaded by tests/, the smoke check
 * and bench.py's CPU-baseline leg as the checker; never by the product.
 *
 * What it restates (reference file:line):
 *   - gate coefficients as the BasicGates constructors compute them
 *     (basic_gates.hpp:341-1408, scalar branches);
 *   - the functor arithmetic on base[b0 << s0 + b1 << s1]
 *     (same lines, scalar branches; AVX-512 branches are not the oracle);
 *   - StateVector::apply: every base index with all control bits 1 and all
 *     target bits 0 (state_vector.hpp:402-510);
 *   - gather_and_execute_on_multi: per part, inner state over the part's
 *     qubits ordered by slot (+ slots 0..3 with opt_slots), gather / apply /
 *     scatter for every outer offset (execute.hpp:318-470,
 *     state_vector.hpp:617-673);
 *   - SvSimMPI::gather_qubits + gather_slots bit permutation
 *     (svsim-mpi.hpp:123-173, mpi_redistributer.hpp:17-33,265-344);
 *   - probability (state_vector.hpp:897-923), norm (63-72).
 * Amplitudes are interleaved complex128, index bit s = slot s.
 */
#include <complex.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "hisv.h"

typedef double complex cplx;

#define PI 3.14159265358979323846          /* types.hpp:19 */
#define PI_BY_2 1.57079632679489661923     /* types.hpp:20 */
#define INV_SQRT_2 0.707106781186547524401 /* types.hpp:23 */

/* A constructed gate: the coefficients the reference's constructor stores. */
typedef struct {
  int type;
  cplx c[16];
  int nc, nt;
  int controls[HS_MAX_CONTROLS];
  int targets[HS_MAX_TARGETS];
} pgate;

static cplx par(const hs_gate* g, int i) { return g->params[2 * i] + I * g->params[2 * i + 1]; }

/* RX(theta): cos_ = cos(theta/2), sin_ = i sin(theta/2)  (basic_gates.hpp:343-347) */
static void rx_coef(cplx th, cplx* c) {
  c[0] = ccos(th / 2.0);
  c[1] = I * csin(th / 2.0);
}
/* RY(theta): cos(theta/2), sin(theta/2)  (basic_gates.hpp:401-405) */
static void ry_coef(cplx th, cplx* c) {
  c[0] = ccos(th / 2.0);
  c[1] = csin(th / 2.0);
}
/* RI(theta): exp(-i theta/2)  (basic_gates.hpp:460-463) */
static void ri_coef(cplx th, cplx* c) { c[0] = cexp(-I * th / 2.0); }
/* RZ(theta) == U1: exp(-i theta/2), exp(+i theta/2)  (basic_gates.hpp:515-519,571) */
static void rz_coef(cplx th, cplx* c) {
  c[0] = cexp(-I * th / 2.0);
  c[1] = cexp(I * th / 2.0);
}
/* *Frac(numerator, power): theta = -pi * numerator / 2^(power-1), unsigned
 * arithmetic as in basic_gates.hpp:732-733 (power-1 wraps for power == 0). */
static double frac_angle(uint32_t num, uint32_t power) {
  return -PI * (double)num / pow(2.0, (double)(uint32_t)(power - 1u));
}

/* Build the coefficient set of a gate (the constructor step). Returns 0 or -1. */
static int construct(const hs_gate* g, pgate* p) {
  memset(p, 0, sizeof(*p));
  p->type = g->type;
  p->nc = g->num_controls;
  p->nt = g->num_targets;
  if (p->nc < 0 || p->nc > HS_MAX_CONTROLS || p->nt < 1 || p->nt > HS_MAX_TARGETS) return -1;
  memcpy(p->controls, g->controls, sizeof(p->controls));
  memcpy(p->targets, g->targets, sizeof(p->targets));
  switch (g->type) {
    case HS_GATE_I: case HS_GATE_X: case HS_GATE_Y: case HS_GATE_Z: case HS_GATE_H:
    case HS_GATE_S: case HS_GATE_TDG: case HS_GATE_SDG:
      break;
    case HS_GATE_SWAP:
      if (p->nt != 2) return -1;
      break;
    case HS_GATE_T: /* base[1] *= sqrt(1i)  (basic_gates.hpp:297) */
      p->c[0] = csqrt(I);
      break;
    case HS_GATE_RX: rx_coef(par(g, 0), p->c); break;
    case HS_GATE_RY: ry_coef(par(g, 0), p->c); break;
    case HS_GATE_RI: ri_coef(par(g, 0), p->c); break;
    case HS_GATE_RZ: case HS_GATE_U1: rz_coef(par(g, 0), p->c); break;
    case HS_GATE_R1: /* rz_{theta}, ri_{-theta}  (basic_gates.hpp:718) */
      rz_coef(par(g, 0), p->c);
      ri_coef(-par(g, 0), p->c + 2);
      break;
    case HS_GATE_RZFRAC: rz_coef(frac_angle(g->frac_num, g->frac_pow), p->c); break;
    case HS_GATE_RXFRAC: rx_coef(frac_angle(g->frac_num, g->frac_pow), p->c); break;
    case HS_GATE_RYFRAC: ry_coef(frac_angle(g->frac_num, g->frac_pow), p->c); break;
    case HS_GATE_RIFRAC: ri_coef(frac_angle(g->frac_num, g->frac_pow), p->c); break;
    case HS_GATE_R1FRAC: /* rzf_{-numerator, power+1}, rif_{numerator, power+1} (:785) */
      rz_coef(frac_angle(0u - g->frac_num, g->frac_pow + 1u), p->c);
      ri_coef(frac_angle(g->frac_num, g->frac_pow + 1u), p->c + 2);
      break;
    case HS_GATE_C1:
      for (int i = 0; i < 4; ++i) p->c[i] = par(g, i);
      break;
    case HS_GATE_C2: /* the constructor copies c_r0 across row r (basic_gates.hpp:972-987) */
      if (p->nt != 2) return -1;
      for (int r = 0; r < 4; ++r)
        for (int k = 0; k < 4; ++k) p->c[4 * r + k] = par(g, 4 * r);
      break;
    case HS_GATE_U2: { /* basic_gates.hpp:1025-1029 */
      cplx phi = par(g, 0), lam = par(g, 1);
      p->c[0] = INV_SQRT_2 + 0.0 * I;
      p->c[1] = -INV_SQRT_2 * (ccos(lam) + I * csin(lam));
      p->c[2] = INV_SQRT_2 * (ccos(phi) + I * csin(phi));
      p->c[3] = INV_SQRT_2 * (ccos(phi + lam) + I * csin(phi + lam));
      break;
    }
    case HS_GATE_U3: { /* basic_gates.hpp:1044-1052 */
      cplx th = par(g, 0), phi = par(g, 1), lam = par(g, 2);
      p->c[0] = ccos(th / 2.0) * ccos((-phi - lam) / 2.0) +
                (I * ccos(th / 2.0)) * csin((-phi - lam) / 2.0);
      p->c[1] = -csin(th / 2.0) * ccos((-phi + lam) / 2.0) +
                (I * -csin(th / 2.0)) * csin((-phi + lam) / 2.0);
      p->c[2] = csin(th / 2.0) * ccos((phi - lam) / 2.0) +
                (I * csin(th / 2.0)) * csin((phi - lam) / 2.0);
      p->c[3] = ccos(th / 2.0) * ccos((phi + lam) / 2.0) +
                (I * ccos(th / 2.0)) * csin((phi + lam) / 2.0);
      break;
    }
    case HS_GATE_RXX: /* h1..h4 + rz_{theta} (basic_gates.hpp:576) */
      if (p->nt != 2) return -1;
      rz_coef(par(g, 0), p->c);
      break;
    case HS_GATE_RYY: /* rx(pi/2) x2, rx(-pi/2) x2, rz_{theta} (:1097) */
      if (p->nt != 2) return -1;
      rx_coef(PI_BY_2, p->c);
      rx_coef(-PI_BY_2, p->c + 2);
      rz_coef(par(g, 0), p->c + 4);
      break;
    case HS_GATE_RZZ: /* rz_{theta} (:1238) */
      if (p->nt != 2) return -1;
      rz_coef(par(g, 0), p->c);
      break;
    default:
      return -1;
  }
  if (p->nt != 1 && p->type != HS_GATE_SWAP && p->type != HS_GATE_C2 &&
      p->type != HS_GATE_RXX && p->type != HS_GATE_RYY && p->type != HS_GATE_RZZ)
    return -1;
  return 0;
}

/* ---- functor bodies (scalar branches) ------------------------------------ */
static void swap2(cplx* a, cplx* b) {
  cplx t = *a;
  *a = *b;
  *b = t;
}
static void f_h(cplx* b, size_t s) { /* basic_gates.hpp:186-189 */
  cplx v0 = b[0], v1 = b[s];
  b[0] = INV_SQRT_2 * (v0 + v1);
  b[s] = INV_SQRT_2 * (v0 - v1);
}
static void f_rx(cplx* b, size_t s, const cplx* c) { /* :360-363 */
  cplx v0 = b[0], v1 = b[s];
  b[0] = c[0] * v0 - c[1] * v1;
  b[s] = -c[1] * v0 + c[0] * v1;
}
static void f_ry(cplx* b, size_t s, const cplx* c) { /* :419-422 */
  cplx v0 = b[0], v1 = b[s];
  b[0] = c[0] * v0 - c[1] * v1;
  b[s] = c[1] * v0 + c[0] * v1;
}
static void f_ri(cplx* b, size_t s, const cplx* c) { /* :475-478 */
  b[0] = b[0] * c[0];
  b[s] = b[s] * c[0];
}
static void f_rz(cplx* b, size_t s, const cplx* c) { /* :531-535 */
  b[0] = b[0] * c[0];
  b[s] = b[s] * c[1];
}
static void f_c1(cplx* b, size_t s, const cplx* c) { /* :855-858 */
  cplx v0 = b[0], v1 = b[s];
  b[0] = c[0] * v0 + c[1] * v1;
  b[s] = c[2] * v0 + c[3] * v1;
}

/* Apply one constructed gate at base with target slot strides s0 (, s1). */
static void functor(const pgate* p, cplx* b, size_t s0, size_t s1) {
  switch (p->type) {
    case HS_GATE_I: break;
    case HS_GATE_X: swap2(&b[0], &b[s0]); break;                 /* :120 */
    case HS_GATE_Y: {                                            /* :142-145 */
      cplx v0 = b[0], v1 = b[s0];
      b[0] = -I * v1;
      b[s0] = I * v0;
      break;
    }
    case HS_GATE_H: f_h(b, s0); break;
    case HS_GATE_Z: b[s0] = b[s0] * -1.0; break;                 /* :230 */
    case HS_GATE_S: b[s0] = b[s0] * I; break;                    /* :262 */
    case HS_GATE_T: b[s0] = b[s0] * p->c[0]; break;              /* :297 */
    case HS_GATE_SDG: b[s0] = b[s0] * -I; break;                 /* :1379 */
    case HS_GATE_TDG: b[s0] = (INV_SQRT_2 * (1.0 - I)) * b[s0]; break; /* :1338 */
    case HS_GATE_RX: case HS_GATE_RXFRAC: f_rx(b, s0, p->c); break;
    case HS_GATE_RY: case HS_GATE_RYFRAC: f_ry(b, s0, p->c); break;
    case HS_GATE_RI: case HS_GATE_RIFRAC: f_ri(b, s0, p->c); break;
    case HS_GATE_RZ: case HS_GATE_U1: case HS_GATE_RZFRAC: f_rz(b, s0, p->c); break;
    case HS_GATE_R1: case HS_GATE_R1FRAC:                        /* :723-724, 790-791 */
      f_rz(b, s0, p->c);
      f_ri(b, s0, p->c + 2);
      break;
    case HS_GATE_C1: case HS_GATE_U2: case HS_GATE_U3: f_c1(b, s0, p->c); break;
    case HS_GATE_SWAP: swap2(&b[s0], &b[s1]); break;             /* :804-805 */
    case HS_GATE_C2: {                                           /* :992-1004 */
      cplx v[4] = {b[0], b[s1], b[s0], b[s0 + s1]};
      size_t o[4] = {0, s1, s0, s0 + s1};
      for (int r = 0; r < 4; ++r)
        b[o[r]] = p->c[4 * r] * v[0] + p->c[4 * r + 1] * v[1] + p->c[4 * r + 2] * v[2] +
                  p->c[4 * r + 3] * v[3];
      break;
    }
    case HS_GATE_RXX:                                            /* :587-599 */
      f_h(b, s0);
      f_h(b + s1, s0);
      f_h(b, s1);
      f_h(b + s0, s1);
      f_h(b, s1);
      swap2(&b[s0], &b[s0 + s1]);
      f_rz(b, s1, p->c);
      f_rz(b + s0, s1, p->c);
      swap2(&b[s0], &b[s0 + s1]);
      f_h(b, s1);
      f_h(b + s0, s1);
      f_h(b, s0);
      f_h(b + s1, s0);
      break;
    case HS_GATE_RYY:                                            /* :1108-1120 */
      f_rx(b, s0, p->c);
      f_rx(b + s1, s0, p->c);
      f_rx(b, s1, p->c);
      f_rx(b + s0, s1, p->c);
      swap2(&b[s0], &b[s0 + s1]);
      f_rz(b, s1, p->c + 4);
      f_rz(b + s0, s1, p->c + 4);
      swap2(&b[s0], &b[s0 + s1]);
      f_rx(b, s0, p->c + 2);
      f_rx(b + s1, s0, p->c + 2);
      f_rx(b, s1, p->c + 2);
      f_rx(b + s0, s1, p->c + 2);
      break;
    case HS_GATE_RZZ:                                            /* :1249-1252 */
      swap2(&b[s0], &b[s0 + s1]);
      f_rz(b, s1, p->c);
      f_rz(b + s0, s1, p->c);
      swap2(&b[s0], &b[s0 + s1]);
      break;
    default: break;
  }
}

/* Deposit the bits of i into the (ascending) slot positions `slots`. */
static uint64_t deposit(uint64_t i, const int* slots, int ns) {
  uint64_t r = 0;
  for (int j = 0; j < ns; ++j) r |= ((i >> j) & 1ull) << slots[j];
  return r;
}

/* StateVector::apply over an nslots-slot buffer whose qubit q sits in slot
 * q2s[q] (state_vector.hpp:402-457). */
static int apply_on(cplx* sv, int nslots, const int* q2s, const pgate* p) {
  int used[64] = {0};
  int ctl_slots[HS_MAX_CONTROLS], tgt_slots[HS_MAX_TARGETS];
  uint64_t control_offset = 0;
  for (int i = 0; i < p->nc; ++i) {
    int q = p->controls[i];
    if (q < 0 || q >= 64 || q2s[q] < 0) return -1;
    ctl_slots[i] = q2s[q];
    control_offset += 1ull << ctl_slots[i];
  }
  for (int i = 0; i < p->nt; ++i) {
    int q = p->targets[i];
    if (q < 0 || q >= 64 || q2s[q] < 0) return -1;
    tgt_slots[i] = q2s[q];
  }
  for (int i = 0; i < p->nc; ++i) {
    if (used[ctl_slots[i]]) return -1;
    used[ctl_slots[i]] = 1;
  }
  for (int i = 0; i < p->nt; ++i) {
    if (used[tgt_slots[i]]) return -1;
    used[tgt_slots[i]] = 1;
  }
  int loop_slots[64], nl = 0;
  for (int s = 0; s < nslots; ++s)
    if (!used[s]) loop_slots[nl++] = s;
  size_t s0 = (size_t)1 << tgt_slots[0];
  size_t s1 = p->nt > 1 ? (size_t)1 << tgt_slots[1] : 0;
  int64_t count = (int64_t)1 << nl;
#pragma omp parallel for schedule(static) if (count > 4096)
  for (int64_t i = 0; i < count; ++i) {
    uint64_t idx = deposit((uint64_t)i, loop_slots, nl) + control_offset;
    functor(p, sv + idx, s0, s1);
  }
  return 0;
}

static int sort_unique(int* v, int n) {
  for (int i = 1; i < n; ++i)
    for (int j = i; j > 0 && v[j - 1] > v[j]; --j) {
      int t = v[j];
      v[j] = v[j - 1];
      v[j - 1] = t;
    }
  int m = 0;
  for (int i = 0; i < n; ++i)
    if (m == 0 || v[m - 1] != v[i]) v[m++] = v[i];
  return m;
}

/* One part, restating gather_and_execute_on_multi (execute.hpp:318-470) on a
 * state with identity slot map. */
static int run_part(cplx* sv, int n, const pgate* gates, int ng, int opt_slots) {
  int qs[64 + 4 * HS_MAX_TARGETS];
  int nq = 0;
  for (int g = 0; g < ng; ++g) {
    for (int i = 0; i < gates[g].nt; ++i) qs[nq++] = gates[g].targets[i];
    for (int i = 0; i < gates[g].nc; ++i) qs[nq++] = gates[g].controls[i];
    nq = sort_unique(qs, nq);
  }
  if (opt_slots) /* execute.hpp:332-347: add the qubits in slots 0..3 */
    for (int s = 0; s < 4 && s < n; ++s) {
      qs[nq++] = s;
      nq = sort_unique(qs, nq);
    }
  for (int i = 0; i < nq; ++i)
    if (qs[i] < 0 || qs[i] >= n) return -1;
  /* inner slot i <-> ordered qubit qs[i] (state_vector.hpp:683-696) */
  int inner_q2s[64];
  for (int q = 0; q < 64; ++q) inner_q2s[q] = -1;
  for (int i = 0; i < nq; ++i) inner_q2s[qs[i]] = i;
  int outer[64], no = 0, mark[64] = {0};
  for (int i = 0; i < nq; ++i) mark[qs[i]] = 1;
  for (int s = 0; s < n; ++s)
    if (!mark[s]) outer[no++] = s;
  const size_t inner_size = (size_t)1 << nq;
  const int64_t outer_count = (int64_t)1 << no;
  int err = 0;
#pragma omp parallel
  {
    cplx* inner = (cplx*)malloc(inner_size * sizeof(cplx));
#pragma omp for schedule(static)
    for (int64_t o = 0; o < outer_count; ++o) {
      uint64_t off = deposit((uint64_t)o, outer, no);
      for (size_t t = 0; t < inner_size; ++t) inner[t] = sv[off + deposit(t, qs, nq)];
      for (int g = 0; g < ng; ++g) {
        /* gates act on the inner state with no omp nesting */
        const pgate* p = &gates[g];
        int used[64] = {0};
        uint64_t coff = 0;
        int ts[HS_MAX_TARGETS];
        for (int i = 0; i < p->nc; ++i) {
          int s = inner_q2s[p->controls[i]];
          coff += 1ull << s;
          used[s] = 1;
        }
        for (int i = 0; i < p->nt; ++i) {
          ts[i] = inner_q2s[p->targets[i]];
          used[ts[i]] = 1;
        }
        int ls[64], nl = 0;
        for (int s = 0; s < nq; ++s)
          if (!used[s]) ls[nl++] = s;
        size_t s0 = (size_t)1 << ts[0];
        size_t s1 = p->nt > 1 ? (size_t)1 << ts[1] : 0;
        for (uint64_t i = 0; i < (1ull << nl); ++i)
          functor(p, inner + deposit(i, ls, nl) + coff, s0, s1);
      }
      for (size_t t = 0; t < inner_size; ++t) sv[off + deposit(t, qs, nq)] = inner[t];
    }
    free(inner);
  }
  return err;
}

/* ---- exported entry points ------------------------------------------------ */

int port_hs_gate_size(void) { return (int)sizeof(hs_gate); }

/* Gate coefficients as constructed (16 complex, zero-padded); for tests. */
int port_construct(const hs_gate* g, double* coef32) {
  pgate p;
  if (construct(g, &p)) return -1;
  memcpy(coef32, p.c, sizeof(p.c));
  return 0;
}

/* Same contract as ref_run in ref_harness.cpp. */
int port_run(int n, const hs_gate* gates, int num_gates, const int32_t* offs,
             int num_parts, int mode, int opt_slots, int init, double* state) {
  if (n < 1 || n > 40) return -1;
  cplx* sv = (cplx*)state;
  const size_t size = (size_t)1 << n;
  if (!init) {
    memset(sv, 0, size * sizeof(cplx));
    sv[0] = 1.0;
  }
  pgate* pg = (pgate*)malloc(sizeof(pgate) * (num_gates > 0 ? num_gates : 1));
  for (int i = 0; i < num_gates; ++i)
    if (construct(&gates[i], &pg[i])) {
      free(pg);
      return -1;
    }
  int q2s[64];
  for (int q = 0; q < 64; ++q) q2s[q] = q < n ? q : -1;
  int rc = 0;
  if (mode == 0) {
    for (int i = 0; i < num_gates && !rc; ++i) rc = apply_on(sv, n, q2s, &pg[i]);
  } else {
    for (int p = 0; p < num_parts && !rc; ++p)
      rc = run_part(sv, n, pg + offs[p], offs[p + 1] - offs[p], opt_slots);
  }
  free(pg);
  return rc;
}

/* Bit permutation of SvSimMPI::gather_qubits / gather_slots: the slots in
 * proc_slots[0..np) (any order) become the top np index bits in ascending slot
 * order, all other slots keep their order below them
 * (svsim-mpi.hpp:141-152; mpi_redistributer.hpp:17-33). */
int port_gather_slots(const double* in, double* out, int n, const int32_t* proc_slots,
                      int np) {
  int is_proc[64] = {0};
  for (int i = 0; i < np; ++i) {
    if (proc_slots[i] < 0 || proc_slots[i] >= n || is_proc[proc_slots[i]]) return -1;
    is_proc[proc_slots[i]] = 1;
  }
  int src[64], k = 0;
  for (int s = 0; s < n; ++s)
    if (!is_proc[s]) src[k++] = s;
  for (int s = 0; s < n; ++s)
    if (is_proc[s]) src[k++] = s;
  const cplx* a = (const cplx*)in;
  cplx* b = (cplx*)out;
  const int64_t size = (int64_t)1 << n;
#pragma omp parallel for schedule(static) if (size > 65536)
  for (int64_t x = 0; x < size; ++x) {
    uint64_t y = 0;
    for (int j = 0; j < n; ++j) y |= (((uint64_t)x >> src[j]) & 1ull) << j;
    b[y] = a[x];
  }
  return 0;
}

/* probability(qubit, value) (state_vector.hpp:897-923): sum |a|^2 over the
 * amplitudes whose slot bit is 0; value 1 returns 1 - that sum. */
double port_probability(int n, const double* state, int slot, int value) {
  const cplx* a = (const cplx*)state;
  long double p0 = 0;
  for (uint64_t i = 0; i < (1ull << n); ++i)
    if (!((i >> slot) & 1ull)) p0 += (long double)(creal(a[i]) * creal(a[i]) + cimag(a[i]) * cimag(a[i]));
  return value == 0 ? (double)p0 : 1.0 - (double)p0;
}

double port_norm2(int n, const double* state) {
  const cplx* a = (const cplx*)state;
  long double s = 0;
  for (uint64_t i = 0; i < (1ull << n); ++i)
    s += (long double)(creal(a[i]) * creal(a[i]) + cimag(a[i]) * cimag(a[i]));
  return (double)s;
}
