/* classifier.c -- TEST INFRASTRUCTURE ONLY (the checker, never the product):
 * CPU restatement of the classifier's inputs and network, for the parity
 * and gradient tests of the GPU classifier.
 *
 *   or_normalise_rows  Applications/candidate_profiler.C:88-134
 *                      (normalise_series_array), same types and order
 *   or_patch_dm        candidate_profiler.C:232-415 (gen_dm_time_plot with
 *                      do_filter) on the pipeline's prefix sums, candidate DM
 *                      at row 32
 *   or_patch_ft        candidate_profiler.C:136-230 (gen_freq_time_plot)
 *   or_cnn_run         the two-branch CNN (heimdall_multibeam_b200/csrc/
 *                      classifier.cu) forward and backward: sums in double,
 *                      BF16 rounding at the points where the GPU rounds
 *                      (GEMM operands and stored activations). */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "oracle.h"

/* ---- normalise_series_array ---------------------------------------------- */
static int cmp_float(const void* a, const void* b) {
  float x = *(const float*)a, y = *(const float*)b;
  return (x > y) - (x < y);
}

/* k-th smallest of v[0..n) (what std::nth_element leaves at position k) */
static float kth(const float* v, size_t n, size_t k, float* tmp) {
  memcpy(tmp, v, n * sizeof(float));
  qsort(tmp, n, sizeof(float), cmp_float);
  return tmp[k];
}

void or_normalise_rows(float* data, size_t n, size_t nrows) {
  float* tmp = (float*)malloc(n * sizeof(float));
  float* a = (float*)malloc(n * sizeof(float));
  for (size_t r = 0; r < nrows; r++) {
    float* x = data + r * n;
    float median1 = kth(x, n / 2, n / 4, tmp);
    float median2 = kth(x + n / 2, n - n / 2, n / 4, tmp);
    /* (median2 - median1) / (nsamps/2): float divided by size_t -> float */
    double gradient = (double)((median2 - median1) / (float)(n / 2));
    float median0 = (float)((double)median1 - gradient * (double)(n / 4));
    for (size_t j = 0; j < n; j++) {
      float baseline = (float)((double)median0 + (double)j * gradient);
      x[j] = x[j] - baseline;
      a[j] = fabsf(x[j]);
    }
    float mad = kth(a, n, n / 2, tmp);
    float stddev = (float)((double)mad * 1.4826);
    float val = (float)(1.0 / (double)stddev);
    /* a row with zero deviation is set to zero (the reference divides by 0) */
    for (size_t j = 0; j < n; j++) x[j] = stddev > 0.f ? x[j] * val : 0.f;
  }
  free(tmp);
  free(a);
}

/* ---- patches ------------------------------------------------------------- */
void or_patch_dm(const float* scans, size_t pitch, size_t len, size_t ndm, size_t dm,
                 size_t ind, size_t filter, float* out) {
  size_t w = (size_t)1 << filter;
  long long first = (ind > 32 + w / 2) ? (long long)ind - 32 - (long long)(w / 2) : 0;
  for (int r = 0; r < 64; r++) {
    long long d = (long long)dm - 32 + r;
    for (int t = 0; t < 64; t++) {
      long long a = first + t, b = a + (long long)w;
      float v = 0.f;
      if (d >= 0 && d < (long long)ndm && b <= (long long)len) {
        const float* S = scans + (size_t)d * pitch;
        v = S[b] - S[a];
      }
      out[r * 64 + t] = v;
    }
  }
  or_normalise_rows(out, 64, 64);
}

void or_patch_ft(const uint8_t* tf, size_t nsamps, size_t nchans, size_t max_delay,
                 size_t ind, size_t filter, float* out) {
  size_t ts = (size_t)1 << filter;
  size_t in_n = 256 * ts;
  if (in_n < max_delay) {
    size_t delay = 2;
    while (delay < max_delay) delay *= 2;
    in_n = delay;
    ts = in_n / 256;
  }
  long long first = (long long)(ind + max_delay / 2) - (long long)(in_n / 2);
  size_t fs = nchans / 64;
  for (int cs = 0; cs < 64; cs++)
    for (int ti = 0; ti < 256; ti++) {
      float sum = 0.f;
      for (size_t s = 0; s < ts; s++) {
        long long t = first + (long long)ti * (long long)ts + (long long)s;
        int in = t >= 0 && t < (long long)nsamps;
        for (size_t f = 0; f < fs; f++) {
          float x = in ? (float)tf[(size_t)t * nchans + cs * fs + f] : 0.f;
          sum += x / 255.f * 255.f;
        }
      }
      out[cs * 256 + ti] = sum / (float)(ts * fs);
    }
  or_normalise_rows(out, 256, 64);
}

/* ---- the network --------------------------------------------------------- */
float or_bf16(float x) {
  uint32_t u;
  memcpy(&u, &x, 4);
  if ((u & 0x7f800000u) != 0x7f800000u) {  /* finite: round to nearest even */
    u += 0x7fffu + ((u >> 16) & 1u);
    u &= 0xffff0000u;
  } else {
    u &= 0xffff0000u;
  }
  memcpy(&x, &u, 4);
  return x;
}

typedef struct { int ci, co, h, w; } conv_spec;
static const conv_spec kConv[2][3] = {{{1, 8, 64, 64}, {8, 16, 32, 32}, {16, 32, 16, 16}},
                                      {{1, 8, 64, 256}, {8, 16, 32, 128}, {16, 32, 16, 64}}};
#define FEAT 10240
#define HID 16

size_t or_cnn_param_count(void) {
  size_t n = 0;
  for (int b = 0; b < 2; b++)
    for (int l = 0; l < 3; l++) n += (size_t)kConv[b][l].co * kConv[b][l].ci * 9 + kConv[b][l].co;
  return n + (size_t)HID * FEAT + HID + 2 * HID + 2;
}

/* offsets in the flat parameter vector (same layout as the GPU) */
static void offsets(size_t ow[2][3], size_t ob[2][3], size_t* ow1, size_t* ob1, size_t* ow2,
                    size_t* ob2) {
  size_t o = 0;
  for (int b = 0; b < 2; b++)
    for (int l = 0; l < 3; l++) {
      ow[b][l] = o; o += (size_t)kConv[b][l].co * kConv[b][l].ci * 9;
      ob[b][l] = o; o += kConv[b][l].co;
    }
  *ow1 = o; o += (size_t)HID * FEAT;
  *ob1 = o; o += HID;
  *ow2 = o; o += 2 * HID;
  *ob2 = o;
}

/* activations [c][n][h][w] */
static float in_at(const float* x, int c, int nb, int b, int h, int w, int y, int xx) {
  if (y < 0 || y >= h || xx < 0 || xx >= w) return 0.f;
  return x[(((size_t)c * nb + b) * h + y) * w + xx];
}

void or_cnn_run(const float* params, const float* dm_time, const float* freq_time,
                const int* labels, size_t n, float* probs, float* grads, float* loss) {
  size_t ow[2][3], ob[2][3], ow1, ob1, ow2, ob2;
  offsets(ow, ob, &ow1, &ob1, &ow2, &ob2);
  const int nb = (int)n;
  /* BF16 copies of the GEMM weights */
  size_t np = or_cnn_param_count();
  float* wb = (float*)malloc(np * sizeof(float));
  for (size_t i = 0; i < np; i++) wb[i] = or_bf16(params[i]);
  float* act[2][4];   /* act[b][0] = input, act[b][l+1] = pooled output of layer l */
  unsigned char* arg[2][3];
  for (int b = 0; b < 2; b++) {
    const conv_spec* s0 = &kConv[b][0];
    size_t nin = (size_t)nb * s0->h * s0->w;
    act[b][0] = (float*)malloc(nin * sizeof(float));
    const float* src = b == 0 ? dm_time : freq_time;
    /* input values limited to +-16 (the GPU's k_input_bf16) */
    for (size_t i = 0; i < nin; i++) act[b][0][i] = or_bf16(fminf(fmaxf(src[i], -16.f), 16.f));
    for (int l = 0; l < 3; l++) {
      const conv_spec* s = &kConv[b][l];
      int h2 = s->h / 2, w2 = s->w / 2;
      size_t nout = (size_t)s->co * nb * h2 * w2;
      act[b][l + 1] = (float*)malloc(nout * sizeof(float));
      arg[b][l] = (unsigned char*)malloc(nout);
      const float* W = wb + ow[b][l];
      const float* B = params + ob[b][l];
      for (int co = 0; co < s->co; co++)
        for (int bi = 0; bi < nb; bi++)
          for (int y2 = 0; y2 < h2; y2++)
            for (int x2 = 0; x2 < w2; x2++) {
              float best = -INFINITY;
              int bq = 0;
              for (int q = 0; q < 4; q++) {
                int y = 2 * y2 + (q >> 1), x = 2 * x2 + (q & 1);
                double z = 0.0;
                for (int ci = 0; ci < s->ci; ci++)
                  for (int t = 0; t < 9; t++)
                    z += (double)W[(size_t)co * s->ci * 9 + ci * 9 + t] *
                         in_at(act[b][l], ci, nb, bi, s->h, s->w, y + t / 3 - 1, x + t % 3 - 1);
                float v = (float)z + B[co];
                v = v > 0.f ? v : 0.f;
                if (v > best) { best = v; bq = q; }
              }
              size_t i = (((size_t)co * nb + bi) * h2 + y2) * w2 + x2;
              act[b][l + 1][i] = or_bf16(best);
              arg[b][l][i] = (unsigned char)bq;
            }
    }
  }
  /* flatten [n][10240] */
  float* x = (float*)malloc((size_t)nb * FEAT * sizeof(float));
  for (int bi = 0; bi < nb; bi++)
    for (int f = 0; f < FEAT; f++) {
      if (f < 2048) x[(size_t)bi * FEAT + f] = act[0][3][((size_t)(f / 64) * nb + bi) * 64 + f % 64];
      else {
        int g = f - 2048;
        x[(size_t)bi * FEAT + f] = act[1][3][((size_t)(g / 256) * nb + bi) * 256 + g % 256];
      }
    }
  float* h = (float*)malloc((size_t)nb * HID * sizeof(float));
  for (int bi = 0; bi < nb; bi++)
    for (int o = 0; o < HID; o++) {
      double z = 0.0;
      for (int f = 0; f < FEAT; f++) z += (double)wb[ow1 + (size_t)o * FEAT + f] * x[(size_t)bi * FEAT + f];
      float v = (float)z + params[ob1 + o];
      h[bi * HID + o] = v > 0.f ? v : 0.f;
    }
  const float* w2 = params + ow2;
  const float* b2 = params + ob2;
  double lsum = 0.0;
  float* d1s = (float*)malloc(nb * sizeof(float));
  for (int bi = 0; bi < nb; bi++) {
    float l0 = b2[0], l1 = b2[1];
    for (int o = 0; o < HID; o++) { l0 += w2[o] * h[bi * HID + o]; l1 += w2[HID + o] * h[bi * HID + o]; }
    float mx = l0 > l1 ? l0 : l1;
    float e0 = expf(l0 - mx), e1 = expf(l1 - mx);
    float p1 = e1 / (e0 + e1);
    if (probs) probs[bi] = p1;
    if (labels) {
      int y = labels[bi];
      lsum += (mx + logf(e0 + e1) - (y ? l1 : l0)) / nb;
      d1s[bi] = (p1 - (y ? 1.f : 0.f)) / nb;
    }
  }
  if (loss) *loss = (float)lsum;
  if (grads && labels) {
    memset(grads, 0, np * sizeof(float));
    float* dz1 = (float*)malloc((size_t)nb * HID * sizeof(float));  /* BF16-rounded */
    for (int bi = 0; bi < nb; bi++) {
      float d1 = d1s[bi], d0 = -d1;
      grads[ob2] += d0;
      grads[ob2 + 1] += d1;
      for (int o = 0; o < HID; o++) {
        float ho = h[bi * HID + o];
        grads[ow2 + o] += d0 * ho;
        grads[ow2 + HID + o] += d1 * ho;
        float dh = d0 * w2[o] + d1 * w2[HID + o];
        float dz = ho > 0.f ? dh : 0.f;
        grads[ob1 + o] += dz;
        dz1[bi * HID + o] = or_bf16(dz);
      }
    }
    for (int o = 0; o < HID; o++)
      for (int f = 0; f < FEAT; f++) {
        double sacc = 0.0;
        for (int bi = 0; bi < nb; bi++) sacc += (double)dz1[bi * HID + o] * x[(size_t)bi * FEAT + f];
        grads[ow1 + (size_t)o * FEAT + f] = (float)sacc;
      }
    /* dx -> pooled-output gradients of both branches */
    float* dact[2];
    dact[0] = (float*)calloc((size_t)32 * nb * 64, sizeof(float));
    dact[1] = (float*)calloc((size_t)32 * nb * 256, sizeof(float));
    for (int bi = 0; bi < nb; bi++)
      for (int f = 0; f < FEAT; f++) {
        double sacc = 0.0;
        for (int o = 0; o < HID; o++) sacc += (double)wb[ow1 + (size_t)o * FEAT + f] * dz1[bi * HID + o];
        if (f < 2048) dact[0][((size_t)(f / 64) * nb + bi) * 64 + f % 64] = (float)sacc;
        else {
          int g = f - 2048;
          dact[1][((size_t)(g / 256) * nb + bi) * 256 + g % 256] = (float)sacc;
        }
      }
    for (int b = 0; b < 2; b++) {
      float* dcur = dact[b];
      for (int l = 2; l >= 0; l--) {
        const conv_spec* s = &kConv[b][l];
        int h2 = s->h / 2, w2b = s->w / 2;
        size_t npre = (size_t)s->co * nb * s->h * s->w;
        float* dz = (float*)calloc(npre, sizeof(float));  /* BF16-rounded */
        for (int co = 0; co < s->co; co++)
          for (int bi = 0; bi < nb; bi++)
            for (int y = 0; y < s->h; y++)
              for (int xx = 0; xx < s->w; xx++) {
                size_t j = (((size_t)co * nb + bi) * h2 + y / 2) * w2b + xx / 2;
                int q = (y & 1) * 2 + (xx & 1);
                float v = 0.f;
                if (arg[b][l][j] == q && act[b][l + 1][j] > 0.f) v = dcur[j];
                grads[ob[b][l] + co] += v;
                dz[(((size_t)co * nb + bi) * s->h + y) * s->w + xx] = or_bf16(v);
              }
        const float* W = wb + ow[b][l];
        for (int co = 0; co < s->co; co++)
          for (int ci = 0; ci < s->ci; ci++)
            for (int t = 0; t < 9; t++) {
              double sacc = 0.0;
              for (int bi = 0; bi < nb; bi++)
                for (int y = 0; y < s->h; y++)
                  for (int xx = 0; xx < s->w; xx++)
                    sacc += (double)dz[(((size_t)co * nb + bi) * s->h + y) * s->w + xx] *
                            in_at(act[b][l], ci, nb, bi, s->h, s->w, y + t / 3 - 1, xx + t % 3 - 1);
              grads[ow[b][l] + (size_t)co * s->ci * 9 + ci * 9 + t] = (float)sacc;
            }
        if (l > 0) {
          size_t nin = (size_t)s->ci * nb * s->h * s->w;
          float* din = (float*)calloc(nin, sizeof(float));
          for (int ci = 0; ci < s->ci; ci++)
            for (int bi = 0; bi < nb; bi++)
              for (int y = 0; y < s->h; y++)
                for (int xx = 0; xx < s->w; xx++) {
                  double sacc = 0.0;
                  for (int t = 0; t < 9; t++) {
                    int yo = y - t / 3 + 1, xo = xx - t % 3 + 1;
                    if (yo < 0 || yo >= s->h || xo < 0 || xo >= s->w) continue;
                    for (int co = 0; co < s->co; co++)
                      sacc += (double)W[(size_t)co * s->ci * 9 + ci * 9 + t] *
                              dz[(((size_t)co * nb + bi) * s->h + yo) * s->w + xo];
                  }
                  din[(((size_t)ci * nb + bi) * s->h + y) * s->w + xx] = (float)sacc;
                }
          if (dcur != dact[b]) free(dcur);
          dcur = din;
        }
        free(dz);
      }
      if (dcur != dact[b]) free(dcur);
      free(dact[b]);
    }
    free(dz1);
  }
  for (int b = 0; b < 2; b++) {
    for (int l = 0; l < 4; l++) free(act[b][l]);
    for (int l = 0; l < 3; l++) free(arg[b][l]);
  }
  free(x); free(h); free(d1s); free(wb);
}
