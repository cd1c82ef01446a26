// unet_oracle.cpp -- TEST INFRASTRUCTURE ONLY: a CPU restatement of the
// learned preconditioner (3-D U-Net) of moons_b200/csrc/unet.cu, used to
// check the CUDA kernels and the gradients of the training step.
//
// The network has no counterpart in the reference (the reference's
// preconditioners are the Jacobi family of
// code/handwritten/solvers/preconditioners/preconditioners.f90:55-129), so
// this restatement is not pinned against reference outputs ("parity
// unpinned"); it is the definition of the network the CUDA path must
// reproduce.  Tensors are [C][Z][Y][X] (interior only, zero padding outside).
// Every tensor the GPU stores in BF16 (activations, their gradients, the
// convolution weights) is rounded to BF16 here at the same points; sums are
// formed in double.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

namespace {

// exact mode: no BF16 rounding anywhere (used to pin the backward pass
// against finite differences of the loss)
bool g_exact = false;

float bf16r(float x) {  // round to nearest even BF16
  if (g_exact) return x;
  uint32_t u;
  std::memcpy(&u, &x, 4);
  if ((u & 0x7f800000u) == 0x7f800000u) return x;
  const uint32_t lsb = (u >> 16) & 1u;
  u += 0x7fffu + lsb;
  u &= 0xffff0000u;
  float r;
  std::memcpy(&r, &u, 4);
  return r;
}

struct T4 {
  int C = 0, X = 0, Y = 0, Z = 0;
  std::vector<float> v;
  T4() = default;
  T4(int c, int x, int y, int z) : C(c), X(x), Y(y), Z(z), v((size_t)c * x * y * z, 0.f) {}
  float& at(int c, int x, int y, int z) { return v[(((size_t)c * Z + z) * Y + y) * X + x]; }
  float get(int c, int x, int y, int z) const {
    if (x < 0 || y < 0 || z < 0 || x >= X || y >= Y || z >= Z) return 0.f;
    return v[(((size_t)c * Z + z) * Y + y) * X + x];
  }
  void round() {
    for (auto& a : v) a = bf16r(a);
  }
};

T4 cat(const T4& a, const T4& b) {
  T4 o(a.C + b.C, a.X, a.Y, a.Z);
  std::copy(a.v.begin(), a.v.end(), o.v.begin());
  std::copy(b.v.begin(), b.v.end(), o.v.begin() + a.v.size());
  return o;
}

// out[co] = sum_ci,tap W[co][ci][tap] in[ci](v + shift(tap))   (+ bias, ReLU)
T4 conv(const T4& in, const std::vector<float>& W, const float* bias, int cout, bool relu) {
  T4 o(cout, in.X, in.Y, in.Z);
  const int cin = in.C;
  for (int co = 0; co < cout; co++)
    for (int z = 0; z < in.Z; z++)
      for (int y = 0; y < in.Y; y++)
        for (int x = 0; x < in.X; x++) {
          double s = 0.0;
          for (int ci = 0; ci < cin; ci++) {
            const float* w = &W[((size_t)co * cin + ci) * 27];
            for (int dz = 0; dz < 3; dz++)
              for (int dy = 0; dy < 3; dy++)
                for (int dx = 0; dx < 3; dx++)
                  s += (double)w[dz * 9 + dy * 3 + dx] * in.get(ci, x + dx - 1, y + dy - 1, z + dz - 1);
          }
          float r = (float)s;
          if (bias) r += bias[co];
          if (relu) r = std::max(r, 0.f);
          o.at(co, x, y, z) = r;
        }
  return o;
}

// gradient w.r.t. the input of conv: din[ci](u) = sum W[co][ci][tap] dout[co](u - shift(tap))
T4 conv_t(const T4& dout, const std::vector<float>& W, int cin) {
  T4 o(cin, dout.X, dout.Y, dout.Z);
  const int cout = dout.C;
  for (int ci = 0; ci < cin; ci++)
    for (int z = 0; z < dout.Z; z++)
      for (int y = 0; y < dout.Y; y++)
        for (int x = 0; x < dout.X; x++) {
          double s = 0.0;
          for (int co = 0; co < cout; co++) {
            const float* w = &W[((size_t)co * cin + ci) * 27];
            for (int dz = 0; dz < 3; dz++)
              for (int dy = 0; dy < 3; dy++)
                for (int dx = 0; dx < 3; dx++)
                  s += (double)w[dz * 9 + dy * 3 + dx] * dout.get(co, x - dx + 1, y - dy + 1, z - dz + 1);
          }
          o.at(ci, x, y, z) = (float)s;
        }
  return o;
}

// dW[co][ci][tap] = sum_v dout[co](v) in[ci](v + shift(tap)); db[co] = sum_v dout[co](v)
void wgrad(const T4& in, const T4& dout, float* dW, float* db) {
  const int cin = in.C, cout = dout.C;
  for (int co = 0; co < cout; co++) {
    for (int ci = 0; ci < cin; ci++)
      for (int dz = 0; dz < 3; dz++)
        for (int dy = 0; dy < 3; dy++)
          for (int dx = 0; dx < 3; dx++) {
            double s = 0.0;
            for (int z = 0; z < in.Z; z++)
              for (int y = 0; y < in.Y; y++)
                for (int x = 0; x < in.X; x++) {
                  const float g = dout.get(co, x, y, z);
                  if (g != 0.f) s += (double)g * in.get(ci, x + dx - 1, y + dy - 1, z + dz - 1);
                }
            dW[((size_t)co * cin + ci) * 27 + dz * 9 + dy * 3 + dx] = (float)s;
          }
    double s = 0.0;
    for (int z = 0; z < in.Z; z++)
      for (int y = 0; y < in.Y; y++)
        for (int x = 0; x < in.X; x++) s += dout.get(co, x, y, z);
    db[co] = (float)s;
  }
}

T4 pool(const T4& a) {
  T4 o(a.C, a.X / 2, a.Y / 2, a.Z / 2);
  for (int c = 0; c < a.C; c++)
    for (int z = 0; z < o.Z; z++)
      for (int y = 0; y < o.Y; y++)
        for (int x = 0; x < o.X; x++) {
          float s = 0.f;  // the GPU sums the 8 children in FP32 in this order
          for (int k = 0; k < 8; k++) s += a.get(c, 2 * x + (k & 1), 2 * y + ((k >> 1) & 1), 2 * z + (k >> 2));
          o.at(c, x, y, z) = s * 0.125f;
        }
  return o;
}

T4 up(const T4& a) {
  T4 o(a.C, a.X * 2, a.Y * 2, a.Z * 2);
  for (int c = 0; c < a.C; c++)
    for (int z = 0; z < o.Z; z++)
      for (int y = 0; y < o.Y; y++)
        for (int x = 0; x < o.X; x++) o.at(c, x, y, z) = a.get(c, x / 2, y / 2, z / 2);
  return o;
}

struct Net {
  struct L {
    int cin, cout;
    size_t wofs, bofs;
    std::vector<float> wq;  // BF16-rounded weights
  };
  std::vector<L> layers;
  size_t head = 0, n = 0;
  const float* p = nullptr;
  explicit Net(const float* params) : p(params) {
    const int io[14][2] = {{8, 16},   {16, 16}, {16, 32}, {32, 32}, {32, 64},  {64, 64}, {64, 128},
                           {128, 128}, {192, 64}, {64, 64}, {96, 32}, {32, 32}, {48, 16}, {16, 16}};
    size_t o = 0;
    for (auto& q : io) {
      L l;
      l.cin = q[0];
      l.cout = q[1];
      l.wofs = o;
      o += (size_t)l.cin * l.cout * 27;
      l.bofs = o;
      o += l.cout;
      l.wq.assign(params + l.wofs, params + l.wofs + (size_t)l.cin * l.cout * 27);
      for (auto& w : l.wq) w = bf16r(w);
      layers.push_back(std::move(l));
    }
    head = o;
    n = o + 17;
  }
  T4 fwd(int l, const T4& in) const {
    T4 o = conv(in, layers[l].wq, p + layers[l].bofs, layers[l].cout, true);
    o.round();
    return o;
  }
};

struct Acts {
  T4 in, e0a, e0, p1, e1a, e1, p2, e2a, e2, p3, e3a, e3, u2, d2a, d2, u1, d1a, d1, u0, d0a, d0;
  T4 y;  // head output (FP32)
};

double rms_interior(const double* r, int X, int Y, int Z) {
  double s = 0.0;
  for (int z = 1; z <= Z; z++)
    for (int y = 1; y <= Y; y++)
      for (int x = 1; x <= X; x++) {
        const double v = r[x + (size_t)(X + 2) * (y + (size_t)(Y + 2) * z)];
        s += v * v;
      }
  return std::sqrt(s / ((double)X * Y * Z));
}

void forward(const Net& N, int X, int Y, int Z, const double* r, const float* feat, double sinv, Acts& a) {
  a.in = T4(8, X, Y, Z);
  for (int z = 0; z < Z; z++)
    for (int y = 0; y < Y; y++)
      for (int x = 0; x < X; x++) {
        const size_t c = (x + 1) + (size_t)(X + 2) * ((y + 1) + (size_t)(Y + 2) * (z + 1));
        a.in.at(0, x, y, z) = bf16r((float)(r[c] * sinv));
        a.in.at(1, x, y, z) = feat ? bf16r(feat[c]) : 0.f;
      }
  a.e0a = N.fwd(0, a.in);
  a.e0 = N.fwd(1, a.e0a);
  a.p1 = pool(a.e0); a.p1.round();
  a.e1a = N.fwd(2, a.p1);
  a.e1 = N.fwd(3, a.e1a);
  a.p2 = pool(a.e1); a.p2.round();
  a.e2a = N.fwd(4, a.p2);
  a.e2 = N.fwd(5, a.e2a);
  a.p3 = pool(a.e2); a.p3.round();
  a.e3a = N.fwd(6, a.p3);
  a.e3 = N.fwd(7, a.e3a);
  a.u2 = up(a.e3);
  a.d2a = N.fwd(8, cat(a.u2, a.e2));
  a.d2 = N.fwd(9, a.d2a);
  a.u1 = up(a.d2);
  a.d1a = N.fwd(10, cat(a.u1, a.e1));
  a.d1 = N.fwd(11, a.d1a);
  a.u0 = up(a.d1);
  a.d0a = N.fwd(12, cat(a.u0, a.e0));
  a.d0 = N.fwd(13, a.d0a);
  a.y = T4(1, X, Y, Z);
  for (int z = 0; z < Z; z++)
    for (int y = 0; y < Y; y++)
      for (int x = 0; x < X; x++) {
        float s = 0.f;
        for (int c = 0; c < 16; c++) s += N.p[N.head + c] * a.d0.at(c, x, y, z);
        a.y.at(0, x, y, z) = s + N.p[N.head + 16];
      }
}

void mask_by(T4& d, const T4& act) {
  for (size_t i = 0; i < d.v.size(); i++)
    if (!(act.v[i] > 0.f)) d.v[i] = 0.f;
}

T4 split(const T4& a, int c0, int c1) {
  T4 o(c1 - c0, a.X, a.Y, a.Z);
  const size_t vs = (size_t)a.X * a.Y * a.Z;
  std::copy(a.v.begin() + c0 * vs, a.v.begin() + c1 * vs, o.v.begin());
  return o;
}

}  // namespace

extern "C" {

void or_unet_set_exact(int on) { g_exact = on != 0; }

// one layer, same contract as moons_unet_layer_check (inputs and weights
// rounded to BF16; the output is not rounded)
int or_unet_layer(int op, int X, int Y, int Z, int cinA, int cinB, int cout, const float* in, const float* dout,
                  const float* W, const float* bias, int relu, float* out) {
  const int cin = cinA + cinB;
  std::vector<float> wq;
  if (W) wq.assign(W, W + (size_t)cout * cin * 27);
  for (auto& w : wq) w = bf16r(w);
  if (!W && op != 2) return 1;
  const size_t vs = (size_t)X * Y * Z;
  if (op == 0 || op == 2) {
    T4 ti(cin, X, Y, Z);
    for (size_t i = 0; i < (size_t)cin * vs; i++) ti.v[i] = bf16r(in[i]);
    if (op == 0) {
      T4 o = conv(ti, wq, relu ? bias : nullptr, cout, relu != 0);
      std::copy(o.v.begin(), o.v.end(), out);
    } else {
      T4 td(cout, X, Y, Z);
      for (size_t i = 0; i < (size_t)cout * vs; i++) td.v[i] = bf16r(dout[i]);
      wgrad(ti, td, out, out + (size_t)cout * cin * 27);
    }
    return 0;
  }
  if (op == 1) {
    T4 td(cout, X, Y, Z);
    for (size_t i = 0; i < (size_t)cout * vs; i++) td.v[i] = bf16r(dout[i]);
    T4 o = conv_t(td, wq, cin);
    std::copy(o.v.begin(), o.v.end(), out);
    return 0;
  }
  return 1;
}

long long or_unet_nparams() {
  std::vector<float> dummy(2000000, 0.f);
  return (long long)Net(dummy.data()).n;
}

// z = out_scale * rms(r) * y(r / rms(r), feat); r, z cell-centred with ghosts
int or_unet_forward(int X, int Y, int Z, const float* params, double out_scale, const double* r, const float* feat,
                    double* z) {
  Net N(params);
  const double rms = rms_interior(r, X, Y, Z);
  Acts a;
  forward(N, X, Y, Z, r, feat, rms > 0 ? 1.0 / rms : 0.0, a);
  const size_t ncc = (size_t)(X + 2) * (Y + 2) * (Z + 2);
  std::fill(z, z + ncc, 0.0);
  for (int zz = 0; zz < Z; zz++)
    for (int y = 0; y < Y; y++)
      for (int x = 0; x < X; x++)
        z[(x + 1) + (size_t)(X + 2) * ((y + 1) + (size_t)(Y + 2) * (zz + 1))] =
            out_scale * rms * (double)a.y.at(0, x, y, zz);
  return 0;
}

// loss = sum (y - t)^2 / sum t^2 with t = e / (out_scale * rms(r)), and its
// gradient with respect to every parameter (same flat order as the GPU)
int or_unet_loss_grad(int X, int Y, int Z, const float* params, double out_scale, const double* r, const float* feat,
                      const double* e, int kind, const double* kx, const double* ky, const double* kz, double hgrid,
                      double* loss, float* grads) {
  Net N(params);
  const double rms = rms_interior(r, X, Y, Z);
  Acts a;
  forward(N, X, Y, Z, r, feat, rms > 0 ? 1.0 / rms : 0.0, a);
  const double sc = out_scale * rms, inv = sc > 0 ? 1.0 / sc : 0.0;
  T4 t(1, X, Y, Z);
  double T2 = 0.0;
  for (int zz = 0; zz < Z; zz++)
    for (int y = 0; y < Y; y++)
      for (int x = 0; x < X; x++) {
        const float v = (float)(e[(x + 1) + (size_t)(X + 2) * ((y + 1) + (size_t)(Y + 2) * (zz + 1))] * inv);
        t.at(0, x, y, zz) = v;
        T2 += (double)v * v;
      }
  const float T2f = T2 > 0 ? (float)T2 : 1.f;
  std::fill(grads, grads + N.n, 0.f);
  double L = 0.0, gb = 0.0;
  // kind 1 (cosine): L = 1 - y.t / (|y| |t|), dL/dy = ca t + cb y
  double yt = 0.0, yy = 0.0;
  for (size_t i = 0; i < t.v.size(); i++) {
    yt += (double)a.y.v[i] * t.v[i];
    yy += (double)a.y.v[i] * a.y.v[i];
  }
  if (!(yy > 0)) yy = 1.0;
  const double ny = std::sqrt(yy), nt = std::sqrt((double)T2f);
  double ca = -1.0 / (ny * nt), cb = yt / (yy * ny * nt);
  // kind 2: energy norm of the volume-weighted sigma-Laplacian on a uniform
  // mesh (spacing hgrid) with homogeneous Neumann walls:
  // (A y)_c = h * sum over the six faces of k_f (y_nb - y_c), no wall flux
  T4 ay(1, X, Y, Z);
  std::vector<double> rh((size_t)X * Y * Z);
  double ea = 0.0, eB = 0.0, eE = 0.0;
  if (kind == 2) {
    const size_t sx = X + 2, sy = Y + 2;
    for (int zz = 0; zz < Z; zz++)
      for (int y = 0; y < Y; y++)
        for (int x = 0; x < X; x++) {
          const int xi = x + 1, yi = y + 1, zi = zz + 1;  // padded cell indices
          const double yc = a.y.at(0, x, y, zz);
          double v = 0.0;
          if (x > 0) v += kx[xi + (sx + 1) * (yi + sy * zi)] * (a.y.at(0, x - 1, y, zz) - yc);
          if (x < X - 1) v += kx[xi + 1 + (sx + 1) * (yi + sy * zi)] * (a.y.at(0, x + 1, y, zz) - yc);
          if (y > 0) v += ky[xi + sx * (yi + (sy + 1) * zi)] * (a.y.at(0, x, y - 1, zz) - yc);
          if (y < Y - 1) v += ky[xi + sx * (yi + 1 + (sy + 1) * zi)] * (a.y.at(0, x, y + 1, zz) - yc);
          if (zz > 0) v += kz[xi + sx * (yi + sy * zi)] * (a.y.at(0, x, y, zz - 1) - yc);
          if (zz < Z - 1) v += kz[xi + sx * (yi + sy * (zi + 1))] * (a.y.at(0, x, y, zz + 1) - yc);
          ay.at(0, x, y, zz) = (float)(hgrid * v);
          const double rv = r[xi + sx * (yi + sy * zi)] * inv;  // A t = r / s
          rh[((size_t)zz * Y + y) * X + x] = rv;
          ea -= yc * rv;
          eB -= yc * ay.at(0, x, y, zz);
          eE -= t.at(0, x, y, zz) * rv;
        }
    if (!(eB > 0)) eB = 1.0;
    if (!(eE > 0)) eE = 1.0;
    ca = 1.0 / std::sqrt(eB * eE);
    cb = -ea / (eB * std::sqrt(eB) * std::sqrt(eE));
  }
  std::vector<double> gw(16, 0.0);
  T4 dd0(16, X, Y, Z);
  for (int zz = 0; zz < Z; zz++)
    for (int y = 0; y < Y; y++)
      for (int x = 0; x < X; x++) {
        const float d = a.y.at(0, x, y, zz) - t.at(0, x, y, zz);
        float dy;
        if (kind == 1) dy = (float)(ca * t.at(0, x, y, zz) + cb * a.y.at(0, x, y, zz));
        else if (kind == 2) dy = (float)(ca * rh[((size_t)zz * Y + y) * X + x] + cb * ay.at(0, x, y, zz));
        else dy = 2.f * d / T2f;
        L += (double)d * d;
        gb += dy;
        for (int c = 0; c < 16; c++) {
          const float h = a.d0.at(c, x, y, zz);
          gw[c] += (double)dy * h;
          dd0.at(c, x, y, zz) = h > 0.f ? bf16r(params[N.head + c] * dy) : 0.f;
        }
      }
  *loss = kind == 1 ? 1.0 - yt / (ny * nt) : (kind == 2 ? 1.0 - ea / std::sqrt(eB * eE) : L / T2f);
  for (int c = 0; c < 16; c++) grads[N.head + c] = (float)gw[c];
  grads[N.head + 16] = (float)gb;

  auto layer_grads = [&](int l, const T4& in, const T4& dpre) {
    wgrad(in, dpre, grads + N.layers[l].wofs, grads + N.layers[l].bofs);
  };
  auto back = [&](int l, const T4& dpre) {
    T4 o = conv_t(dpre, N.layers[l].wq, N.layers[l].cin);
    o.round();
    return o;
  };
  // dec0b
  layer_grads(13, a.d0a, dd0);
  T4 dd0a = back(13, dd0);
  mask_by(dd0a, a.d0a);
  // dec0a: input cat(u0, e0)
  layer_grads(12, cat(a.u0, a.e0), dd0a);
  T4 dcat0 = back(12, dd0a);
  T4 du0 = split(dcat0, 0, 32), de0 = split(dcat0, 32, 48);
  // up backward -> d1
  auto up_bwd = [](const T4& du, const T4& act) {
    T4 o(du.C, du.X / 2, du.Y / 2, du.Z / 2);
    for (int c = 0; c < o.C; c++)
      for (int z = 0; z < o.Z; z++)
        for (int y = 0; y < o.Y; y++)
          for (int x = 0; x < o.X; x++) {
            float s = 0.f;
            for (int k = 0; k < 8; k++) s += du.get(c, 2 * x + (k & 1), 2 * y + ((k >> 1) & 1), 2 * z + (k >> 2));
            o.at(c, x, y, z) = act.get(c, x, y, z) > 0.f ? bf16r(s) : 0.f;
          }
    return o;
  };
  auto pool_bwd = [](T4& d, const T4& dp, const T4& act) {
    for (int c = 0; c < d.C; c++)
      for (int z = 0; z < d.Z; z++)
        for (int y = 0; y < d.Y; y++)
          for (int x = 0; x < d.X; x++) {
            float& v = d.at(c, x, y, z);
            v = act.get(c, x, y, z) > 0.f ? bf16r(v + 0.125f * dp.get(c, x / 2, y / 2, z / 2)) : 0.f;
          }
  };
  T4 dd1 = up_bwd(du0, a.d1);
  layer_grads(11, a.d1a, dd1);
  T4 dd1a = back(11, dd1);
  mask_by(dd1a, a.d1a);
  layer_grads(10, cat(a.u1, a.e1), dd1a);
  T4 dcat1 = back(10, dd1a);
  T4 du1 = split(dcat1, 0, 64), de1 = split(dcat1, 64, 96);
  T4 dd2 = up_bwd(du1, a.d2);
  layer_grads(9, a.d2a, dd2);
  T4 dd2a = back(9, dd2);
  mask_by(dd2a, a.d2a);
  layer_grads(8, cat(a.u2, a.e2), dd2a);
  T4 dcat2 = back(8, dd2a);
  T4 du2 = split(dcat2, 0, 128), de2 = split(dcat2, 128, 192);
  T4 de3 = up_bwd(du2, a.e3);
  layer_grads(7, a.e3a, de3);
  T4 de3a = back(7, de3);
  mask_by(de3a, a.e3a);
  layer_grads(6, a.p3, de3a);
  T4 dp3 = back(6, de3a);
  pool_bwd(de2, dp3, a.e2);
  layer_grads(5, a.e2a, de2);
  T4 de2a = back(5, de2);
  mask_by(de2a, a.e2a);
  layer_grads(4, a.p2, de2a);
  T4 dp2 = back(4, de2a);
  pool_bwd(de1, dp2, a.e1);
  layer_grads(3, a.e1a, de1);
  T4 de1a = back(3, de1);
  mask_by(de1a, a.e1a);
  layer_grads(2, a.p1, de1a);
  T4 dp1 = back(2, de1a);
  pool_bwd(de0, dp1, a.e0);
  layer_grads(1, a.e0a, de0);
  T4 de0a = back(1, de0);
  mask_by(de0a, a.e0a);
  layer_grads(0, a.in, de0a);
  return 0;
}

// One Adam step (Kingma & Ba 2015, Algorithm 1) on a flat FP32 parameter
// vector, in the form the library's training step applies it: m = b1 m +
// (1-b1) g, v = b2 v + (1-b2) g^2, w -= lr (m c1) / (sqrt(v c2) + eps) with
// the bias corrections c1 = 1/(1-b1^t), c2 = 1/(1-b2^t); FP32 throughout.
void or_unet_adam(float* w, const float* g, float* m, float* v, long long n, float lr, int t) {
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  const float c1 = 1.f / (1.f - std::pow(b1, (float)t));
  const float c2 = 1.f / (1.f - std::pow(b2, (float)t));
  for (long long i = 0; i < n; i++) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    w[i] -= lr * (mi * c1) / (std::sqrt(vi * c2) + eps);
  }
}

}  // extern "C"
