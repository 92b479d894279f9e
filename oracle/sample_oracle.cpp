// ORACLE -- test infrastructure only. CPU restatement of the headless views
// of the field, used by tests/ as the checker and never linked into the
// product library.
//
// Followed (reference paths):
//   common_d3_tree_sample.wgsl   sampleAtLevel / sampleDense / sampleTreeAtMost:
//                                nearest cell of the finest level present,
//                                g = floor((p + 1/2) 2^m), owning block g/(2RB)
//   common_d3_resample.wgsl      volCentre = origin + (v + 1/2) h - 1/2,
//                                texel (ux, uy, uz, rho), the level written
//   common_d3_render_slice.wgsl  planeDims, planePoint, rotateUVW, dPlane,
//                                magColor, uvToPlane, fs_main
//   common_vortcolor.wgsl        vorticityTone / vorticityColor
// The pixel grid is the fragment grid of a full-screen quad: uv at pixel
// centres, uv.y = 1 on the top row; colours are rounded to 8 bits. All in
// f32, each operation rounded on its own (built with -ffp-contract=off).

#include <algorithm>
#include <cmath>
#include <cstdint>

namespace {

struct View {
  int nx, ny, nz, levels, rb, fb, t3;
  const float *mac;        // 4 per L0 cell
  const float *macp;       // 4 per pool cell
  const int32_t *block_slot;
};

struct Smp {
  float v[4];
  int level;
  float c[3];
};

int twrap(int v, int n) {
  const int r = v % n;
  return r < 0 ? r + n : r;
}

Smp sample_tree(const View &t, const float p[3], int mmax) {
  Smp o;
  if (std::min(mmax, t.levels) >= 1) {
    const int dims[3] = {2 * t.nx, 2 * t.ny, 2 * t.nz};
    const int rb2 = 2 * t.rb;
    float gf[3];
    int g[3], b[3];
    for (int a = 0; a < 3; ++a) {
      gf[a] = std::floor((p[a] + 0.5f) * 2.f);
      g[a] = twrap((int)gf[a], dims[a]);
      b[a] = g[a] / rb2;
    }
    const int nbx = t.nx / t.rb, nby = t.ny / t.rb;
    const int slot = t.block_slot[(b[2] * nby + b[1]) * nbx + b[0]];
    if (slot >= 0) {
      const int64_t cell = (int64_t)slot * t.t3 + ((int64_t)(g[2] - b[2] * rb2 + 2) * t.fb + (g[1] - b[1] * rb2 + 2)) * t.fb +
                           (g[0] - b[0] * rb2 + 2);
      for (int k = 0; k < 4; ++k) o.v[k] = t.macp[4 * cell + k];
      o.level = 1;
      for (int a = 0; a < 3; ++a) o.c[a] = (gf[a] + 0.5f) / 2.f - 0.5f;
      return o;
    }
  }
  int c[3];
  for (int a = 0; a < 3; ++a) {
    o.c[a] = std::floor(p[a] + 0.5f);
  }
  c[0] = twrap((int)o.c[0], t.nx);
  c[1] = twrap((int)o.c[1], t.ny);
  c[2] = twrap((int)o.c[2], t.nz);
  const int64_t cell = ((int64_t)c[2] * t.ny + c[1]) * t.nx + c[0];
  for (int k = 0; k < 4; ++k) o.v[k] = t.mac[4 * cell + k];
  o.level = 0;
  return o;
}

struct Slice {
  int axis, slice, mode, rot;
  float u_scale, v_scale, vort_scale, vort_gamma;
  int W, H;
  float off[3];
};

void rot3(int axis, const float in[3], float out[3]) {
  if (axis == 0) { out[0] = in[1]; out[1] = in[2]; out[2] = in[0]; }
  else if (axis == 1) { out[0] = in[2]; out[1] = in[0]; out[2] = in[1]; }
  else { out[0] = in[0]; out[1] = in[1]; out[2] = in[2]; }
}

struct PS {
  float uvw[3], ab[3];
  int level;
};

PS sample_plane(const View &t, const Slice &s, float a, float b, int mmax) {
  const float sl = (float)s.slice;
  float p[3];
  if (s.axis == 0) { p[0] = sl; p[1] = a; p[2] = b; }
  else if (s.axis == 1) { p[0] = b; p[1] = sl; p[2] = a; }
  else { p[0] = a; p[1] = b; p[2] = sl; }
  for (int k = 0; k < 3; ++k) p[k] = p[k] + s.off[k];
  const Smp q = sample_tree(t, p, mmax);
  PS o;
  const float u[3] = {q.v[1], q.v[2], q.v[3]};
  rot3(s.axis, u, o.uvw);
  rot3(s.axis, q.c, o.ab);
  o.level = q.level;
  return o;
}

float d_plane(const View &t, const Slice &s, float pa, float pb, int comp, int axis, int mstart) {
  int m = mstart;
  float h = 1.f / (float)(1 << m);
  PS plus = sample_plane(t, s, pa + (axis == 0 ? h : 0.f), pb + (axis == 1 ? h : 0.f), m);
  PS minus = sample_plane(t, s, pa - (axis == 0 ? h : 0.f), pb - (axis == 1 ? h : 0.f), m);
  for (int it = 0; it < t.levels && plus.level != minus.level; ++it) {
    m = std::min(plus.level, minus.level);
    h = 1.f / (float)(1 << m);
    plus = sample_plane(t, s, pa + (axis == 0 ? h : 0.f), pb + (axis == 1 ? h : 0.f), m);
    minus = sample_plane(t, s, pa - (axis == 0 ? h : 0.f), pb - (axis == 1 ? h : 0.f), m);
  }
  const float dx = plus.ab[axis] - minus.ab[axis];
  if (std::fabs(dx) < 1e-6f * std::max(h, 1e-6f)) return 0.f;
  return (plus.uvw[comp] - minus.uvw[comp]) / dx;
}

float mix1(float a, float b, float t) { return a * (1.f - t) + b * t; }

float smooth(float e0, float e1, float x) {
  const float t = std::min(std::max((x - e0) / (e1 - e0), 0.f), 1.f);
  return t * t * (3.f - 2.f * t);
}

void mag_color(float v, float rgb[3]) {
  const float c = std::min(std::max(v, 0.f), 1.f);
  const float lo0[3] = {0.05f, 0.05f, 0.12f}, lo1[3] = {0.1f, 0.65f, 0.75f}, hi[3] = {1.0f, 0.92f, 0.35f};
  const float s0 = smooth(0.f, 0.55f, c), s1 = smooth(0.55f, 1.f, c);
  for (int k = 0; k < 3; ++k) rgb[k] = mix1(mix1(lo0[k], lo1[k], s0), hi[k], s1);
}

void vort_color(float omega, float scale, float gamma, float rgb[3]) {
  const float a = std::fabs(omega) * scale;
  const float compressed = a / (1.f + a);
  const float mag = std::pow(compressed, gamma);
  const float val = omega >= 0.f ? mag : -mag;
  const float bg[3] = {0.05f, 0.05f, 0.1f}, pos[3] = {1.0f, 0.3f, 0.2f}, neg[3] = {0.2f, 0.5f, 1.0f};
  for (int k = 0; k < 3; ++k) rgb[k] = val > 0.f ? mix1(bg[k], pos[k], val) : mix1(bg[k], neg[k], -val);
}

uint8_t unorm8(float x) {
  const float c = std::min(std::max(x, 0.f), 1.f);
  return (uint8_t)std::nearbyint(c * 255.f);
}

}  // namespace

extern "C" {

// The resampled box: 4 f32 per voxel (ux, uy, uz, rho), x fastest, and the
// answering level per voxel (may be NULL).
int oracle_tree_resample(int nx, int ny, int nz, const float *mac, int levels, const float *macp,
                         const int32_t *block_slot, int rb, int fb, const float *origin, const int32_t *shape,
                         const float *h, float *out, uint8_t *level) {
  const View t{nx, ny, nz, levels, rb, fb, fb * fb * fb, mac, macp, block_slot};
  for (int z = 0; z < shape[2]; ++z)
    for (int y = 0; y < shape[1]; ++y)
      for (int x = 0; x < shape[0]; ++x) {
        const int v[3] = {x, y, z};
        float p[3];
        for (int a = 0; a < 3; ++a) p[a] = origin[a] + ((float)v[a] + 0.5f) * h[a] - 0.5f;
        const Smp s = sample_tree(t, p, levels);
        const int64_t idx = ((int64_t)z * shape[1] + y) * shape[0] + x;
        out[4 * idx] = s.v[1];
        out[4 * idx + 1] = s.v[2];
        out[4 * idx + 2] = s.v[3];
        out[4 * idx + 3] = s.v[0];
        if (level) level[idx] = (uint8_t)s.level;
      }
  return 0;
}

// One slice picture, RGBA8, rows top to bottom. params = {axis, slice, mode,
// rot, W, H}; scales = {u_scale, v_scale, vort_scale, vort_gamma}; off = the
// window's view offset.
int oracle_tree_slice(int nx, int ny, int nz, const float *mac, int levels, const float *macp,
                      const int32_t *block_slot, int rb, int fb, const int32_t *params, const float *scales,
                      const float *off, uint8_t *rgba) {
  const View t{nx, ny, nz, levels, rb, fb, fb * fb * fb, mac, macp, block_slot};
  const Slice s{params[0], params[1], params[2], params[3], scales[0], scales[1], scales[2], scales[3],
                params[4], params[5], {off[0], off[1], off[2]}};
  const int nd[3] = {nx, ny, nz};
  const float dx = (float)nd[(s.axis + 1) % 3], dy = (float)nd[(s.axis + 2) % 3];
  for (int py = 0; py < s.H; ++py)
    for (int px = 0; px < s.W; ++px) {
      const float u = ((float)px + 0.5f) / (float)s.W;
      const float v = 1.f - ((float)py + 0.5f) / (float)s.H;
      float pa, pb;
      if (s.rot == 1) { pa = (1.f - v) * dx - 0.5f; pb = (1.f - u) * dy - 0.5f; }
      else if (s.rot == 2) { pa = (1.f - u) * dx - 0.5f; pb = v * dy - 0.5f; }
      else if (s.rot == 3) { pa = v * dx - 0.5f; pb = u * dy - 0.5f; }
      else { pa = u * dx - 0.5f; pb = (1.f - v) * dy - 0.5f; }
      const PS q = sample_plane(t, s, pa, pb, levels);
      float rgb[3];
      if (s.mode == 1) {
        const float omega = d_plane(t, s, pa, pb, 1, 0, q.level) - d_plane(t, s, pa, pb, 0, 1, q.level);
        vort_color(omega / std::max(s.v_scale, 1e-12f), s.vort_scale, s.vort_gamma, rgb);
      } else if (s.mode == 2) {
        vort_color(q.uvw[2] / std::max(s.u_scale, 1e-9f), s.vort_scale, s.vort_gamma, rgb);
      } else {
        const float len = std::sqrt(q.uvw[0] * q.uvw[0] + q.uvw[1] * q.uvw[1] + q.uvw[2] * q.uvw[2]);
        mag_color(len / std::max(s.u_scale, 1e-9f), rgb);
      }
      uint8_t *o = rgba + 4 * ((int64_t)py * s.W + px);
      o[0] = unorm8(rgb[0]);
      o[1] = unorm8(rgb[1]);
      o[2] = unorm8(rgb[2]);
      o[3] = 255;
    }
  return 0;
}

}  // extern "C"
