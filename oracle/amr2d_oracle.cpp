// ORACLE -- test infrastructure only. CPU restatement of the reference's 2D
// block-structured AMR macro-step (levels = 2, `interp` interface), used by
// the tests as the checker for the device implementation.
//
// Followed (reference paths):
//   main-cylinder-amr.js:1831-1889  dispatchMacroStep order: refine round every
//                                   REFINE_EVERY, finest-level force, S_Advance
//   amr2d-gpu.mjs:984-1011          makeRefineRound order
//   amr2d-gpu.mjs:1120-1160         S_Advance (interp): fill L1 ring from L0,
//                                   L0 step, two L1 substeps, average into L0
//   amr2d-gpu.mjs:262-302           writePoolInitialState (free list 0..n-1)
//   amr_step1.wgsl:335-597          pool step (DIRECT_GHOST, COLLIDE_RING = 1,
//                                   CELL_CENTRE_AFFINE = 1, tau_f = 2 tau_c - 1/2)
//   common_interp_kernel.wgsl       interpCell (ring: same-level neighbour copy
//                                   else parent interpolation; whole tile on
//                                   activation)
//   common_interp.wgsl, common_interp_parent_pool.wgsl  bilinear rho, u, fneq
//                                   with the post-collision factor
//   common_average.wgsl             4-child restriction
//   amr_criterion_pool.wgsl,        max |discrete curl| per child quadrant
//   common_criterion.wgsl
//   amr_manage_pool.wgsl            decide (nearBodyBox or vorticity ladder),
//                                   DET_SLOTS coarsen and refine by quads
//   common_geometry.wgsl:230-290    nearBodyBox branch and bound
//   amr_force1.wgsl:350-496         finest-level force with dx weights
//   amr2d-gpu.mjs:1096-1124         S_AdvanceExplode: explode, two substeps
//                                   (the ring advects, COLLIDE_RING = 0),
//                                   coalesce into L0's time-t buffer, the L0
//                                   step, the restriction into L0's new buffer
//   amr_explode.wgsl:132-203        ring <- L0 at t (linear term, in-orphans)
//   amr_coalesce.wgsl:91-172        covered L0 cells <- mean of 4 fine cells;
//                                   out/in-orphan balance at the seam
//   amr_force1.wgsl:241-256         RING_FREE_FORCE gather (explode path)
//
// The topology path (criterion, decide, grant) is always evaluated in f32 with
// every operation rounded, which is what the device does, so the two agree
// bit for bit on the same velocity field. The vorticity decision is the exact
// comparison max|curl| >= 2^REFINE_THRESH (the monotone form of the
// reference's log2 ladder).

#include "common.h"

namespace {
using namespace oracle;

template <class R> struct Amr2D {
  lbm_amr2d_config c{};
  int W = 0, H = 0, RB = 8, G = 2, FB = 20, RB2 = 16, NBX = 0, NBY = 0, PNX = 0, PNY = 0, S = 0;
  int64_t N0 = 0, N1 = 0;  // root cells, pool cells
  std::vector<R> f0[2], vel0, f1[2], vel1;
  int cur = 0;
  std::vector<int32_t> blockSlot, slotToBlock, parentSlot, freeList, activeList;
  int32_t freeCount = 0;
  std::vector<uint32_t> want, newly;
  std::vector<float> crit;
  int64_t step = 0;
  double force[4] = {0, 0, 0, 0};
  lbm_config root{};

  explicit Amr2D(const lbm_amr2d_config &cfg) : c(cfg) {
    W = c.nx; H = c.ny; RB = c.rb; G = 2; RB2 = 2 * RB; FB = RB2 + 2 * G;
    NBX = W / RB; NBY = H / RB; PNX = W / RB2; PNY = H / RB2; S = c.max_slots;
    N0 = (int64_t)W * H; N1 = (int64_t)S * FB * FB;
    for (auto &v : f0) v.assign(9 * N0, R(0));
    vel0.assign(2 * N0, R(0));
    for (auto &v : f1) v.assign(9 * N1, R(0));
    vel1.assign(2 * N1, R(0));
    blockSlot.assign(NBX * NBY, -1);
    slotToBlock.assign(S, -1);
    parentSlot.assign(S, 0);
    freeList.resize(S / 4);
    for (int i = 0; i < S / 4; ++i) freeList[i] = i;
    freeCount = S / 4;
    want.assign(NBX * NBY, 0);
    newly.assign(S, 0);
    crit.assign(NBX * NBY, 0.f);
    std::memset(&root, 0, sizeof(root));
    root.q = 9; root.nx = W; root.ny = H; root.nz = 1; root.tau = c.tau;
    root.force[0] = c.force[0]; root.force[1] = c.force[1];
    root.has_body = 1; root.use_bounceback = c.use_bounceback; root.solid_eq = c.solid_eq;
    root.chi_eps = c.k_eps; root.sponge_w = c.sponge_w;
    root.sponge_u[0] = c.sponge_u[0]; root.sponge_u[1] = c.sponge_u[1];
    root.body = c.body;
  }

  R tau_c() const { return R(c.tau); }
  R tau_f() const { return R(2) * R(c.tau) - R(0.5); }
  const R dxL = R(0.5);
  R cco() const { return R(0.5) * (R(1) - dxL); }  // CELL_CENTRE_AFFINE
  R pos(int bcoord, int fcoord) const { return R(bcoord * RB) - cco() + dxL * R(fcoord - G); }
  int64_t cell1(int slot, int fx, int fy) const { return (int64_t)slot * FB * FB + (int64_t)fy * FB + fx; }
  static int wrapi(int v, int n) { return ((v % n) + n) % n; }
  bool covered(int x, int y) const { return blockSlot[(wrapi(y, H) / RB) * NBX + wrapi(x, W) / RB] >= 0; }
  int64_t rcell(int x, int y) const { return (int64_t)wrapi(y, H) * W + wrapi(x, W); }
  bool explode_mode() const { return c.iface == 1; }

  // amr_explode.wgsl: the ring of every active tile from L0 at time t.
  void explode(const std::vector<R> &fr, std::vector<R> &dst) {
    const Tables &T = tables(9);
    const int NFX = 2 * W, NFY = 2 * H;
    for (int s : activeList) {
      const int bid = slotToBlock[s], bx = bid % NBX, by = bid / NBX;
      for (int fy = 0; fy < FB; ++fy)
        for (int fx = 0; fx < FB; ++fx) {
          if (fx >= G && fx < G + RB2 && fy >= G && fy < G + RB2) continue;
          const int gx = wrapi(bx * RB2 + fx - G, NFX), gy = wrapi(by * RB2 + fy - G, NFY);
          const int vx = gx / 2, vy = gy / 2;
          if (covered(vx, vy)) continue;
          const int64_t vc = rcell(vx, vy);
          R fv[9];
          for (int i = 0; i < 9; ++i) fv[i] = fr[i * N0 + vc];
          bool okx = false, oky = false;
          if (c.explode_linear) {
            okx = !covered(vx - 1, vy) && !covered(vx + 1, vy);
            oky = !covered(vx, vy - 1) && !covered(vx, vy + 1);
          }
          const R dx = (R(gx - 2 * vx) - R(0.5)) * R(0.5), dy = (R(gy - 2 * vy) - R(0.5)) * R(0.5);
          const int64_t cell = cell1(s, fx, fy);
          for (int i = 0; i < 9; ++i) {
            const int ex = T.ex[i], ey = T.ey[i];
            R o;
            if (covered(vx + ex, vy + ey)) {
              o = fv[i];
              if (c.explode_linear && (okx || oky)) {
                R Gx = 0, Gy = 0;
                if (okx) Gx = R(0.5) * (fr[i * N0 + rcell(vx + 1, vy)] - fr[i * N0 + rcell(vx - 1, vy)]);
                if (oky) Gy = R(0.5) * (fr[i * N0 + rcell(vx, vy + 1)] - fr[i * N0 + rcell(vx, vy - 1)]);
                const R ef = (Gx * R(ex) + Gy * R(ey)) / R(ex * ex + ey * ey);
                Gx -= R(ex) * ef;
                Gy -= R(ey) * ef;
                o += dx * Gx + dy * Gy;
              }
            } else {
              const int dgx = wrapi(gx + ex, NFX), dgy = wrapi(gy + ey, NFY);
              const bool into = covered(dgx / 2, dgy / 2) && dgx / RB2 == bx && dgy / RB2 == by;
              o = into ? fv[i] : R(0);
            }
            dst[i * N1 + cell] = o;
          }
        }
    }
  }

  // amr_coalesce.wgsl: covered L0 cells (time-t buffer) take the mean of the
  // four fine cells the L0 step will pull; unrefined cells at the seam get
  // the out-orphans less the in-orphans explode injected.
  void coalesce(const std::vector<R> &fp, std::vector<R> &fr) {
    const Tables &T = tables(9);
    const int NFX = 2 * W, NFY = 2 * H;
    std::vector<R> out = fr;
    for (int cy = 0; cy < H; ++cy)
      for (int cx = 0; cx < W; ++cx) {
        const int64_t cc = rcell(cx, cy);
        if (covered(cx, cy)) {
          const int cbx = cx / RB, cby = cy / RB;
          const int cs = blockSlot[cby * NBX + cbx];
          for (int i = 0; i < 9; ++i) {
            const int tx = cx + T.ex[i], ty = cy + T.ey[i];
            if (covered(tx, ty)) continue;
            R sum = 0;
            for (int k = 0; k < 4; ++k) {
              const int px = tx * 2 + (k & 1), py = ty * 2 + (k >> 1);
              sum += fp[i * N1 + cell1(cs, px - cbx * RB2 + G, py - cby * RB2 + G)];
            }
            out[i * N0 + cc] = sum * R(0.25);
          }
          continue;
        }
        bool nearc = false;
        for (int i = 1; i < 9; ++i) nearc = nearc || covered(cx + T.ex[i], cy + T.ey[i]);
        if (!nearc) continue;
        for (int i = 1; i < 9; ++i) {
          const int ex = T.ex[i], ey = T.ey[i];
          if (covered(cx + ex, cy + ey)) continue;
          R sum = 0, nin = 0;
          for (int k = 0; k < 4; ++k) {
            const int ox = k & 1, oy = k >> 1;
            const int pux = (cx + ex) * 2 + ox, puy = (cy + ey) * 2 + oy;
            const int qx = wrapi(pux - ex, NFX), qy = wrapi(puy - ey, NFY);
            const int qbx = qx / RB2, qby = qy / RB2;
            const int qs = blockSlot[qby * NBX + qbx];
            if (qs >= 0) sum += fp[i * N1 + cell1(qs, qx - qbx * RB2 + G + ex, qy - qby * RB2 + G + ey)];
            const int chx = wrapi(cx * 2 + ox + ex, NFX), chy = wrapi(cy * 2 + oy + ey, NFY);
            if (covered(chx / 2, chy / 2)) nin += R(1);
          }
          const R own = fr[i * N0 + cc];
          const R net = sum - nin * own;
          if (net != R(0)) out[i * N0 + cc] = own + net * R(0.25);
        }
      }
    fr.swap(out);
  }

  R feq(R rho, R ux, R uy, int i) const {
    const Tables &T = tables(9);
    R eu = R(T.ex[i]) * ux + R(T.ey[i]) * uy;
    return R(T.w[i]) * rho * (R(1) + R(3) * eu + R(4.5) * eu * eu - R(1.5) * (ux * ux + uy * uy));
  }

  // ---- topology (always f32, every operation rounded) ----------------------

  static float phi2f(float px, float py, const lbm_body &b, float Wf, float Hf) {
    return phi2<float>(px, py, b, Wf, Hf);
  }

  bool near_body_box(float cx, float cy, float half) const {
    const float SQRT2_UP = 1.4142136f;
    const float margin = c.refine_margin, la = c.refine_lookahead;
    lbm_body fut = c.body;
    fut.theta = c.body.theta + c.body.wz * la;
    struct E { float x, y, h; int d; };
    E st[16];
    int sp = 0;
    st[sp++] = {cx, cy, half, 3};
    while (sp > 0) {
      E e = st[--sp];
      float now = phi2f(e.x, e.y, c.body, (float)W, (float)H);
      float fu = phi2f(e.x - c.body.vx * la, e.y - c.body.vy * la, fut, (float)W, (float)H);
      float phi = std::fmin(now, fu);
      if (phi - e.h * SQRT2_UP > margin) continue;
      if (phi <= margin) return true;
      if (e.d == 0) return true;
      float hh = e.h * 0.5f;
      for (int i = 0; i < 4; ++i)
        st[sp++] = {e.x + ((i & 1) ? hh : -hh), e.y + ((i & 2) ? hh : -hh), hh, e.d - 1};
    }
    return false;
  }

  void criterion() {
    // Root taps are periodic across tiles (GHOST == 0 branch).
    std::vector<float> v(2 * N0);
    for (int64_t k = 0; k < 2 * N0; ++k) v[k] = (float)vel0[k];
    for (int by = 0; by < NBY; ++by)
      for (int bx = 0; bx < NBX; ++bx) {
        float m = 0.f;
        for (int ly = 0; ly < RB; ++ly)
          for (int lx = 0; lx < RB; ++lx) {
            const int x = bx * RB + lx, y = by * RB + ly;
            const int xp = (x + 1) % W, xm = (x + W - 1) % W, yp = (y + 1) % H, ym = (y + H - 1) % H;
            const float a = v[2 * ((int64_t)y * W + xp) + 1], b = v[2 * ((int64_t)y * W + xm) + 1];
            const float cc = v[2 * ((int64_t)yp * W + x)], d = v[2 * ((int64_t)ym * W + x)];
            const float om = (a - b) * 0.5f - (cc - d) * 0.5f;
            m = std::fmax(m, std::fabs(om));
          }
        crit[by * NBX + bx] = m;
      }
  }

  void decide() {
    const double thr = std::exp2((double)c.refine_thresh);
    for (int pb = 0; pb < PNX * PNY; ++pb) {
      const int bxP = pb % PNX, byP = pb / PNX;
      float mc = 0.f;
      for (int q = 0; q < 4; ++q) mc = std::fmax(mc, crit[(byP * 2 + (q >> 1)) * NBX + bxP * 2 + (q & 1)]);
      const bool vort = c.refine_thresh <= 1.0f && std::fmax((double)mc, 1e-6) >= thr;
      const float half = (float)RB;
      const float ctr_x = (float)(bxP * RB2) + half - 0.5f, ctr_y = (float)(byP * RB2) + half - 0.5f;
      const bool w = near_body_box(ctr_x, ctr_y, half) || vort;
      for (int q = 0; q < 4; ++q) want[(byP * 2 + (q >> 1)) * NBX + bxP * 2 + (q & 1)] = w ? 1u : 0u;
    }
  }

  void coarsen_refine() {
    int32_t count = freeCount;
    for (int s = 0; s < S; s += 4) {
      const int b = slotToBlock[s];
      if (b < 0 || want[b]) continue;
      freeList[count++] = s / 4;
      for (int q = 0; q < 4; ++q) {
        const int bb = slotToBlock[s + q];
        if (bb >= 0) blockSlot[bb] = -1;
        slotToBlock[s + q] = -1;
      }
    }
    for (int ps = 0; ps < PNX * PNY; ++ps) {  // root slot == root block
      const int bxP = ps % PNX, byP = ps / PNX;
      const int b0 = (byP * 2) * NBX + bxP * 2;
      if (blockSlot[b0] >= 0 || !want[b0]) continue;
      if (count <= 0) continue;  // pool exhausted: stays coarse
      count -= 1;
      const int quad = freeList[count];
      for (int qy = 0; qy < 2; ++qy)
        for (int qx = 0; qx < 2; ++qx) {
          const int slot = quad * 4 + qx + 2 * qy;
          const int bid = (byP * 2 + qy) * NBX + bxP * 2 + qx;
          blockSlot[bid] = slot;
          slotToBlock[slot] = bid;
          parentSlot[slot] = ps;
          newly[slot] = 1;
        }
    }
    freeCount = count;
    activeList.clear();
    for (int s = 0; s < S; ++s)
      if (slotToBlock[s] >= 0) activeList.push_back(s);
  }

  // ---- transfers ------------------------------------------------------------

  struct Sample { R rho, ux, uy, fneq[9]; };

  Sample sample_parent(int gx, int gy) const {
    gx = ((gx % W) + W) % W;
    gy = ((gy % H) + H) % H;
    const int64_t cell = (int64_t)gy * W + gx;
    const Tables &T = tables(9);
    R f[9], rho = 0, ux = 0, uy = 0;
    for (int i = 0; i < 9; ++i) {
      f[i] = f0[cur][i * N0 + cell];
      rho += f[i]; ux += f[i] * R(T.ex[i]); uy += f[i] * R(T.ey[i]);
    }
    ux /= std::fmax(rho, R(1e-6)); uy /= std::fmax(rho, R(1e-6));
    Sample s{rho, ux, uy, {}};
    for (int i = 0; i < 9; ++i) s.fneq[i] = f[i] - feq(rho, ux, uy, i);
    return s;
  }

  void interp_cell(int slot, int bx, int by, int fx, int fy) {
    const R px = R(bx * RB) - R(0.25) + R(0.5) * R(fx - G);
    const R py = R(by * RB) - R(0.25) + R(0.5) * R(fy - G);
    const int x0 = (int)std::floor(px), y0 = (int)std::floor(py);
    const R tx = px - R(x0), ty = py - R(y0);
    const Sample s00 = sample_parent(x0, y0), s10 = sample_parent(x0 + 1, y0);
    const Sample s01 = sample_parent(x0, y0 + 1), s11 = sample_parent(x0 + 1, y0 + 1);
    const R w00 = (R(1) - tx) * (R(1) - ty), w10 = tx * (R(1) - ty), w01 = (R(1) - tx) * ty, w11 = tx * ty;
    const R rho = w00 * s00.rho + w10 * s10.rho + w01 * s01.rho + w11 * s11.rho;
    const R ux = w00 * s00.ux + w10 * s10.ux + w01 * s01.ux + w11 * s11.ux;
    const R uy = w00 * s00.uy + w10 * s10.uy + w01 * s01.uy + w11 * s11.uy;
    const R tc = tau_c(), tf = R(2) * tc - R(0.5);
    const R resc = R(0.5) * (tf - R(1)) / (tc - R(1));
    const int64_t cell = cell1(slot, fx, fy);
    for (int i = 0; i < 9; ++i) {
      const R fneq = w00 * s00.fneq[i] + w10 * s10.fneq[i] + w01 * s01.fneq[i] + w11 * s11.fneq[i];
      f1[0][i * N1 + cell] = feq(rho, ux, uy, i) + resc * fneq;
    }
  }

  void init_fill() {
    for (int s : activeList) {
      if (!newly[s]) continue;
      const int b = slotToBlock[s], bx = b % NBX, by = b / NBX;
      for (int fy = 0; fy < FB; ++fy)
        for (int fx = 0; fx < FB; ++fx) interp_cell(s, bx, by, fx, fy);
    }
  }

  void ghost_fill() {
    for (int s : activeList) {
      const int b = slotToBlock[s], bx = b % NBX, by = b / NBX;
      const int bxm = (bx + NBX - 1) % NBX, bxp = (bx + 1) % NBX, bym = (by + NBY - 1) % NBY, byp = (by + 1) % NBY;
      for (int fy = 0; fy < FB; ++fy)
        for (int fx = 0; fx < FB; ++fx) {
          const bool inX = fx >= G && fx < G + RB2, inY = fy >= G && fy < G + RB2;
          if (inX && inY) continue;
          int ns = -1, nfx = fx, nfy = fy;
          if (inY && fx < G) { ns = blockSlot[by * NBX + bxm]; nfx = fx + RB2; }
          else if (inY && fx >= G + RB2) { ns = blockSlot[by * NBX + bxp]; nfx = fx - RB2; }
          else if (inX && fy < G) { ns = blockSlot[bym * NBX + bx]; nfy = fy + RB2; }
          else if (inX && fy >= G + RB2) { ns = blockSlot[byp * NBX + bx]; nfy = fy - RB2; }
          else if (fx < G && fy < G) { ns = blockSlot[bym * NBX + bxm]; nfx = fx + RB2; nfy = fy + RB2; }
          else if (fx >= G + RB2 && fy < G) { ns = blockSlot[bym * NBX + bxp]; nfx = fx - RB2; nfy = fy + RB2; }
          else if (fx < G && fy >= G + RB2) { ns = blockSlot[byp * NBX + bxm]; nfx = fx + RB2; nfy = fy - RB2; }
          else { ns = blockSlot[byp * NBX + bxp]; nfx = fx - RB2; nfy = fy - RB2; }
          if (ns >= 0) {
            const int64_t dst = cell1(s, fx, fy), src = cell1(ns, nfx, nfy);
            for (int i = 0; i < 9; ++i) f1[0][i * N1 + dst] = f1[0][i * N1 + src];
          } else {
            interp_cell(s, bx, by, fx, fy);
          }
        }
    }
  }

  void substep(const std::vector<R> &fin, std::vector<R> &fout) {
    const Tables &T = tables(9);
    const lbm_body &b = c.body;
    const R CS2 = R(1) / R(3), fW = R(W), fH = R(H);
    const R omg = R(1) / tau_f();
    const R eps = R(c.k_eps) * dxL;
    for (int s : activeList) {
      const int bid = slotToBlock[s], bx = bid % NBX, by = bid / NBX;
      const int bxm = (bx + NBX - 1) % NBX, bxp = (bx + 1) % NBX, bym = (by + NBY - 1) % NBY, byp = (by + 1) % NBY;
      for (int fy = 0; fy < FB; ++fy)
        for (int fx = 0; fx < FB; ++fx) {
          const int offX = fx <= G ? -1 : (fx + 1 >= G + RB2 ? 1 : 0);
          const int offY = fy <= G ? -1 : (fy + 1 >= G + RB2 ? 1 : 0);
          const int cxb = offX > 0 ? bxp : (offX < 0 ? bxm : bx);
          const int cyb = offY > 0 ? byp : (offY < 0 ? bym : by);
          const int nbrX = offX ? blockSlot[by * NBX + cxb] : -1;
          const int nbrY = offY ? blockSlot[cyb * NBX + bx] : -1;
          const int nbrXY = (offX && offY) ? blockSlot[cyb * NBX + cxb] : -1;
          const int64_t cell = cell1(s, fx, fy);
          const R px = pos(bx, fx), py = pos(by, fy);
          R wx = std::fmod(px, fW); if (wx < R(0)) wx += fW;
          R wy = std::fmod(py, fH); if (wy < R(0)) wy += fH;
          const R rx = wrapd(px - R(b.cx), fW), ry = wrapd(py - R(b.cy), fH);
          const R usx = R(b.vx) - R(b.wz) * ry, usy = R(b.vy) + R(b.wz) * rx;
          const R phi = phi2<R>(px, py, b, fW, fH);
          R f[9];
          for (int i = 0; i < 9; ++i) {
            if (c.use_bounceback) {
              const R sxp = pos(bx, fx - T.ex[i]), syp = pos(by, fy - T.ey[i]);
              if (phi2<R>(sxp, syp, b, fW, fH) < R(0)) {
                const R corr = R(2) * R(T.w[i]) * (R(T.ex[i]) * usx + R(T.ey[i]) * usy) / CS2;
                f[i] = fin[T.opp[i] * N1 + cell] + corr;
                continue;
              }
            }
            int sx = fx - T.ex[i], sy = fy - T.ey[i], src = s;
            const int ox = (sx < G || sx >= G + RB2) ? offX : 0;
            const int oy = (sy < G || sy >= G + RB2) ? offY : 0;
            const int ns = (ox && oy) ? nbrXY : (ox ? nbrX : (oy ? nbrY : -1));
            if (ns >= 0) { src = ns; sx -= ox * RB2; sy -= oy * RB2; }
            sx = std::min(std::max(sx, 0), FB - 1);
            sy = std::min(std::max(sy, 0), FB - 1);
            f[i] = fin[i * N1 + cell1(src, sx, sy)];
          }
          R rho = 0, uxs = 0, uys = 0;
          for (int i = 0; i < 9; ++i) { rho += f[i]; uxs += f[i] * R(T.ex[i]); uys += f[i] * R(T.ey[i]); }
          const R den = std::fmax(rho, R(1e-6));
          uxs /= den; uys /= den;
          const R chi = c.use_bounceback ? R(0) : chi_of(phi, eps);
          const R Fx = rho * chi * (usx - uxs) + R(c.force[0]);
          const R Fy = rho * chi * (usy - uys) + R(c.force[1]);
          const R ux = uxs + Fx / (R(2) * den), uy = uys + Fy / (R(2) * den);
          const R usq = ux * ux + uy * uy;
          vel1[2 * cell] = ux; vel1[2 * cell + 1] = uy;
          if (explode_mode() && !(fx >= G && fx < G + RB2 && fy >= G && fy < G + RB2)) {
            for (int i = 0; i < 9; ++i) fout[i * N1 + cell] = f[i];  // COLLIDE_RING = 0
            continue;
          }
          const R dx = std::fmin(wx, fW - R(1) - wx), dy = std::fmin(wy, fH - R(1) - wy);
          const R sw = sponge(std::fmin(dx, dy), R(c.sponge_w));
          const bool solid = c.solid_eq && c.use_bounceback && phi < R(0);
          const R SUX = R(c.sponge_u[0]), SUY = R(c.sponge_u[1]);
          for (int i = 0; i < 9; ++i) {
            const R exf = R(T.ex[i]), eyf = R(T.ey[i]), w = R(T.w[i]);
            R o;
            if (solid) {
              o = feq(R(1), usx, usy, i);
            } else {
              const R eu = exf * ux + eyf * uy;
              const R fe = w * rho * (R(1) + R(3) * eu + R(4.5) * eu * eu - R(1.5) * usq);
              const R t2 = (exf * ux + eyf * uy) * R(9);
              const R Si = (R(1) - R(0.5) * omg) * w *
                           (((exf - ux) * R(3) + t2 * exf) * Fx + ((eyf - uy) * R(3) + t2 * eyf) * Fy);
              const R fc = f[i] - omg * (f[i] - fe) + Si;
              const R euf = exf * SUX + eyf * SUY;
              const R ft = w * (R(1) + R(3) * euf + R(4.5) * euf * euf - R(1.5) * (SUX * SUX + SUY * SUY));
              o = fc * (R(1) - sw) + ft * sw;
            }
            fout[i * N1 + cell] = o;
          }
        }
    }
  }

  void average(std::vector<R> &dst) {
    const Tables &T = tables(9);
    const R tc = tau_c(), tf = tau_f();
    const R resc = R(2) * (tc - R(1)) / (tf - R(1));
    for (int s : activeList) {
      const int bid = slotToBlock[s], bx = bid % NBX, by = bid / NBX;
      for (int ly = 0; ly < RB; ++ly)
        for (int lx = 0; lx < RB; ++lx) {
          const int fx0 = G + 2 * lx, fy0 = G + 2 * ly;
          const int64_t ch[4] = {cell1(s, fx0, fy0), cell1(s, fx0 + 1, fy0), cell1(s, fx0, fy0 + 1),
                                 cell1(s, fx0 + 1, fy0 + 1)};
          R fc[4][9], rc[4], uxc[4], uyc[4];
          R rs = 0, rxs = 0, rys = 0;
          for (int k = 0; k < 4; ++k) {
            R rho = 0, ux = 0, uy = 0;
            for (int i = 0; i < 9; ++i) {
              fc[k][i] = f1[0][i * N1 + ch[k]];
              rho += fc[k][i]; ux += fc[k][i] * R(T.ex[i]); uy += fc[k][i] * R(T.ey[i]);
            }
            ux /= std::fmax(rho, R(1e-6)); uy /= std::fmax(rho, R(1e-6));
            rc[k] = rho; uxc[k] = ux; uyc[k] = uy;
            rs += rho; rxs += rho * ux; rys += rho * uy;
          }
          const R ra = rs * R(0.25);
          const R den = std::fmax(rs, R(1e-6));
          const R uxa = rxs / den, uya = rys / den;
          const int64_t pc = (int64_t)(by * RB + ly) * W + (bx * RB + lx);
          for (int i = 0; i < 9; ++i) {
            R sum = 0;
            for (int k = 0; k < 4; ++k) sum += fc[k][i] - feq(rc[k], uxc[k], uyc[k], i);
            dst[i * N0 + pc] = feq(ra, uxa, uya, i) + resc * (sum * R(0.25));
          }
        }
    }
  }

  void force_l1() {
    const Tables &T = tables(9);
    const lbm_body &b = c.body;
    const R CS2 = R(1) / R(3), fW = R(W), fH = R(H);
    const R eps = R(c.k_eps) * dxL;
    double acc[4] = {0, 0, 0, 0};
    for (int s : activeList) {
      const int bid = slotToBlock[s], bx = bid % NBX, by = bid / NBX;
      for (int fy = G; fy < G + RB2; ++fy)
        for (int fx = G; fx < G + RB2; ++fx) {
          const R px = pos(bx, fx), py = pos(by, fy);
          const R phi = phi2<R>(px, py, b, fW, fH);
          const int64_t cell = cell1(s, fx, fy);
          R fxb = 0, fyb = 0, tz = 0;
          const R rx = wrapd(px - R(b.cx), fW), ry = wrapd(py - R(b.cy), fH);
          const R usx = R(b.vx) - R(b.wz) * ry, usy = R(b.vy) + R(b.wz) * rx;
          if (c.use_bounceback) {
            if (phi >= R(0)) {
              for (int i = 0; i < 9; ++i) {
                const R sxp = pos(bx, fx - T.ex[i]), syp = pos(by, fy - T.ey[i]);
                if (phi2<R>(sxp, syp, b, fW, fH) < R(0)) {
                  const R fo = f1[0][T.opp[i] * N1 + cell];
                  const R corr = R(2) * R(T.w[i]) * (R(T.ex[i]) * usx + R(T.ey[i]) * usy) / CS2;
                  fxb += -R(T.ex[i]) * (R(2) * fo + corr) * dxL;
                  fyb += -R(T.ey[i]) * (R(2) * fo + corr) * dxL;
                }
              }
              tz = rx * fyb - ry * fxb;
            }
          } else {
            const R chi = chi_of(phi, eps);
            if (chi >= R(1e-6)) {
              R rho = 0, ux = 0, uy = 0;
              for (int i = 0; i < 9; ++i) {
                const int sx0 = fx - T.ex[i], sy0 = fy - T.ey[i];
                const int sx = std::min(std::max(sx0, 0), FB - 1);
                const int sy = std::min(std::max(sy0, 0), FB - 1);
                int64_t src = cell1(s, sx, sy);
                if (explode_mode()) {  // RING_FREE_FORCE: resolve as the step's gather does
                  const int ox = sx0 >= G + RB2 ? 1 : (sx0 < G ? -1 : 0);
                  const int oy = sy0 >= G + RB2 ? 1 : (sy0 < G ? -1 : 0);
                  if (ox || oy) {
                    const int ns = blockSlot[((by + oy + NBY) % NBY) * NBX + (bx + ox + NBX) % NBX];
                    if (ns >= 0) src = cell1(ns, sx0 - ox * RB2, sy0 - oy * RB2);
                  }
                }
                const R v = f1[0][i * N1 + src];
                rho += v; ux += v * R(T.ex[i]); uy += v * R(T.ey[i]);
              }
              ux /= std::fmax(rho, R(1e-6)); uy /= std::fmax(rho, R(1e-6));
              const R Fx = rho * chi * (usx - ux), Fy = rho * chi * (usy - uy);
              fxb = -Fx * dxL; fyb = -Fy * dxL;
              tz = rx * fyb - ry * fxb;
            }
          }
          const R v3[3] = {fxb, fyb, tz};
          for (int k = 0; k < 3; ++k) {
            if (std::isfinite((double)v3[k])) acc[k] += (double)v3[k];
            else acc[3] += 1;
          }
        }
    }
    for (int k = 0; k < 4; ++k) force[k] = acc[k];
  }

  void refine_round() {
    std::fill(newly.begin(), newly.end(), 0u);
    criterion();
    std::fill(want.begin(), want.end(), 0u);
    decide();
    coarsen_refine();
    init_fill();
  }

  void macro_step() {
    if (c.auto_refine && step % c.refine_every == 0) refine_round();
    ++step;
    force_l1();
    if (explode_mode()) {
      explode(f0[cur], f1[0]);
      substep(f1[0], f1[1]);
      substep(f1[1], f1[0]);
      coalesce(f1[0], f0[cur]);
      std::vector<double> mac(4 * N0);
      step2<R>(root, f0[cur], f0[1 - cur], mac.data());
      for (int64_t k = 0; k < N0; ++k) { vel0[2 * k] = R(mac[4 * k + 1]); vel0[2 * k + 1] = R(mac[4 * k + 2]); }
      average(f0[1 - cur]);
      cur = 1 - cur;
      return;
    }
    ghost_fill();
    std::vector<double> mac(4 * N0);
    step2<R>(root, f0[cur], f0[1 - cur], mac.data());
    for (int64_t k = 0; k < N0; ++k) { vel0[2 * k] = R(mac[4 * k + 1]); vel0[2 * k + 1] = R(mac[4 * k + 2]); }
    substep(f1[0], f1[1]);
    substep(f1[1], f1[0]);
    average(f0[1 - cur]);
    cur = 1 - cur;
  }
};

struct Handle {
  int fp32 = 0;
  Amr2D<double> *d = nullptr;
  Amr2D<float> *f = nullptr;
};

template <class A> void write_root(A &a, const double *f, const double *vel) {
  for (int64_t k = 0; k < 9 * a.N0; ++k) a.f0[a.cur][k] = f[k];
  for (int64_t k = 0; k < 2 * a.N0; ++k) a.vel0[k] = vel[k];
}

template <class A> void read_all(A &a, double *f0, double *vel0, double *f1, double *vel1, int32_t *topo,
                                 float *crit, double *force) {
  if (f0) for (int64_t k = 0; k < 9 * a.N0; ++k) f0[k] = (double)a.f0[a.cur][k];
  if (vel0) for (int64_t k = 0; k < 2 * a.N0; ++k) vel0[k] = (double)a.vel0[k];
  if (f1) for (int64_t k = 0; k < 9 * a.N1; ++k) f1[k] = (double)a.f1[0][k];
  if (vel1) for (int64_t k = 0; k < 2 * a.N1; ++k) vel1[k] = (double)a.vel1[k];
  if (topo) {
    // block_slot | slot_to_block | free_list | free_count | n_active | active | want
    int32_t *p = topo;
    for (int v : a.blockSlot) *p++ = v;
    for (int v : a.slotToBlock) *p++ = v;
    for (int v : a.freeList) *p++ = v;
    *p++ = a.freeCount;
    *p++ = (int32_t)a.activeList.size();
    for (int k = 0; k < a.S; ++k) *p++ = k < (int)a.activeList.size() ? a.activeList[k] : -1;
    for (uint32_t v : a.want) *p++ = (int32_t)v;
  }
  if (crit) for (size_t k = 0; k < a.crit.size(); ++k) crit[k] = a.crit[k];
  if (force) for (int k = 0; k < 4; ++k) force[k] = a.force[k];
}

}  // namespace

extern "C" {

void *oracle_amr2d_create(const lbm_amr2d_config *c, int fp32) {
  Handle *h = new Handle();
  h->fp32 = fp32;
  if (fp32) h->f = new Amr2D<float>(*c);
  else h->d = new Amr2D<double>(*c);
  return h;
}

void oracle_amr2d_destroy(void *hp) {
  Handle *h = (Handle *)hp;
  delete h->d;
  delete h->f;
  delete h;
}

void oracle_amr2d_write_root(void *hp, const double *f, const double *vel) {
  Handle *h = (Handle *)hp;
  if (h->fp32) write_root(*h->f, f, vel); else write_root(*h->d, f, vel);
}

void oracle_amr2d_step(void *hp, int n) {
  Handle *h = (Handle *)hp;
  for (int k = 0; k < n; ++k) {
    if (h->fp32) h->f->macro_step(); else h->d->macro_step();
  }
}

// Topology alone from a given root velocity (f32 semantics): criterion,
// decide, coarsen/refine. The state's topology arrays advance.
void oracle_amr2d_refine_from_vel(void *hp, const float *vel) {
  Handle *h = (Handle *)hp;
  auto go = [&](auto &a) {
    for (int64_t k = 0; k < 2 * a.N0; ++k) a.vel0[k] = vel[k];
    std::fill(a.newly.begin(), a.newly.end(), 0u);
    a.criterion();
    std::fill(a.want.begin(), a.want.end(), 0u);
    a.decide();
    a.coarsen_refine();
  };
  if (h->fp32) go(*h->f); else go(*h->d);
}

// Loads a topology state (block_slot, slot_to_block, free_list, free_count);
// the active list is rebuilt from slot_to_block.
void oracle_amr2d_set_topology(void *hp, const int32_t *block_slot, const int32_t *slot_to_block,
                               const int32_t *free_list, int32_t free_count) {
  Handle *h = (Handle *)hp;
  auto go = [&](auto &a) {
    for (size_t k = 0; k < a.blockSlot.size(); ++k) a.blockSlot[k] = block_slot[k];
    for (int k = 0; k < a.S; ++k) a.slotToBlock[k] = slot_to_block[k];
    for (int k = 0; k < a.S / 4; ++k) a.freeList[k] = free_list[k];
    a.freeCount = free_count;
    a.activeList.clear();
    for (int k = 0; k < a.S; ++k)
      if (a.slotToBlock[k] >= 0) a.activeList.push_back(k);
  };
  if (h->fp32) go(*h->f); else go(*h->d);
}

void oracle_amr2d_read(void *hp, double *f0, double *vel0, double *f1, double *vel1, int32_t *topo, float *crit,
                       double *force) {
  Handle *h = (Handle *)hp;
  if (h->fp32) read_all(*h->f, f0, vel0, f1, vel1, topo, crit, force);
  else read_all(*h->d, f0, vel0, f1, vel1, topo, crit, force);
}

}  // extern "C"
