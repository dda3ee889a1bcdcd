// The finite-rate source generated for one mechanism and compiled at a
// case's set-up, as the reference renders its chemistry kernels with the
// species indices and constants as literals
// (peregrine/simulator/mixture/chemistry/kernels/finiterate.mako, compiled
// at run time, peregrine/backend/cuda/compiler.py).
//
// The table-driven kernel (chem.cuh: ratestate, oneway, fold; k_source)
// walks the mechanism's columns at run time; its per-reaction species
// lookups index the rate state's arrays, which then live in local memory.
// Here each reaction becomes straight-line code with its species as literal
// indices, so the rate state, the concentrations and the production rates
// are registers.  The arithmetic of every step is the table-driven kernel's,
// in its order, each constant a hexadecimal literal of the same double.
//
// The kernel reads the leading fields of the library's block record (six
// ints, then the cell count and the offset: BlockHead below, checked against
// BlockDev by the host), the tile table of a packed launch, Q, the state's T
// and the table log's and exp's tables by pointer; it writes dQ as k_source
// does.  NVRTC is opened at run time, so the library needs it only where a
// case asks for the generated kernel.
#include <dlfcn.h>

#include <cmath>
#include <cstdio>
#include <string>
#include <vector>

#include "layout.cuh"
#include "rategen.h"

namespace pgb {

namespace {

std::string lit(double x) {
  char b[64];
  std::snprintf(b, sizeof b, "%a", x);
  return std::string("(") + b + ")";
}
std::string I(int k) { return std::to_string(k); }

const char *kPrelude = R"PGB(
struct alignas(8) TileRef { int x, y; };
struct BlockHead { int nx, ny, nz, X, Y, Z; long long vol, cv; };
struct MathTables { double logtab[128], rcptab[128], exptab[64]; };

__device__ __forceinline__ double tlog(const double x, const MathTables *__restrict__ mt) {
  long long bits = __double_as_longlong(x);
  const int expo = (int)((bits >> 52) & 0x7ff) - 1022;
  const int bin = (int)((bits >> 45) & 127);
  bits = (bits & 0x000fffffffffffffLL) | 0x3fe0000000000000LL;
  const double mant = __longlong_as_double(bits);
  const double u = mant * __ldg(&mt->rcptab[bin]) - 1.0;
  double series = 0.2;
  series = series * u - 0.25;
  series = series * u + 1.0 / 3.0;
  series = series * u - 0.5;
  series = series * u + 1.0;
  return expo * 0x1.62e42fefa39efp-1 + __ldg(&mt->logtab[bin]) + u * series;
}

__device__ __forceinline__ double texp(const double v, const MathTables *__restrict__ mt) {
  const double t = v * 0x1.71547652b82fep+6 + 6755399441055744.0;
  long long bits = __double_as_longlong(t);
  const int kexp = (int)bits, nexp = kexp >> 6;
  const double kd = t - 6755399441055744.0;
  const double r = (v - kd * 0x1.62e42fef00000p-7) - kd * 0x1.473de6af278edp-40;
  double series = 1.0 / 120.0;
  series = series * r + 1.0 / 24.0;
  series = series * r + 1.0 / 6.0;
  series = series * r + 0.5;
  series = series * r + 1.0;
  series = series * r + 1.0;
  const double m = __ldg(&mt->exptab[kexp & 63]) * series;
  bits = __double_as_longlong(m);
  bits += (long long)(nexp > -1022 ? nexp : -1022) << 52;
  return __longlong_as_double(bits);
}
)PGB";

// Troe's broadening added to ln k (chem.cuh: troeblend)
void troe(const Mech &m, const Rxn &r, std::string &o) {
  o += "    {\n      double lfc;\n";
  if (r.nfcent == 0) {
    o += "      lfc = " + lit(m.lfcfloor) + ";\n";
  } else {
    o += "      const double tf = (logT - " + lit(m.troeuc) + ") * " + lit(m.troeuhinv) + ";\n";
    o += "      lfc = " + lit(m.lfcpoly[r.troe][m.nlfc - 1]) + ";\n";
    for (int k = m.nlfc - 2; k >= 0; k--) o += "      lfc = lfc * tf + " + lit(m.lfcpoly[r.troe][k]) + ";\n";
  }
  o += "      const double C = -0.4 - 0.67 * lfc, N = 0.75 - 1.27 * lfc;\n"
       "      const double A = logpr * 0.4342944819032518 + C, B = N - 0.14 * A, B2 = B * B;\n"
       "      lk += lfc * B2 / (B2 + A * A) * 2.302585092994046;\n    }\n";
}

// one reaction's rate of progress added into omega (chem.cuh: oneway, fold)
void reaction(const Mech &m, const Rxn &r, int k, std::string &o) {
  const std::string clamp = lit(m.expclamp);
  const bool falloff = r.kind >= 2, thirdbody = r.kind != 0;
  o += "  {  // reaction " + I(k) + "\n";
  o += "    double lk = " + lit(r.logA) + ";\n";
  if (r.b != 0.0) o += "    lk += " + lit(r.b) + " * logT;\n";
  if (r.EaR != 0.0) o += "    lk -= " + lit(r.EaR) + " * Tinv;\n";
  if (falloff) {
    o += "    double logpr = logtb" + I(r.tb) + " + " + lit(r.logprA) + ";\n";
    if (r.prb != 0.0) o += "    logpr += " + lit(r.prb) + " * logT;\n";
    if (r.prEaR != 0.0) o += "    logpr -= " + lit(r.prEaR) + " * Tinv;\n";
  }
  if (r.product) {
    if (falloff)
      o += "    double pfac;\n    {\n      const double pr = texp(fmin(logpr, " + clamp +
           "), mt);\n      pfac = pr / (1.0 + pr);\n    }\n";
    if (r.kind == 3) troe(m, r, o);
    o += "    double xk = lk;\n";
    for (int j = 0; j < r.nreact; j++) o += "    xk -= " + lit(r.reactnu[j]) + " * gRT" + I(r.reactsp[j]) + ";\n";
    o += "    double K = texp(fmin(xk, " + clamp + "), mt);\n";
    if (thirdbody && !falloff) o += "    K *= ctb" + I(r.tb) + ";\n";
    if (falloff) o += "    K *= pfac;\n";
    o += "    double fwd = K;\n";
    for (int j = 0; j < r.nreact; j++)
      for (int q = 0; q < (int)r.reactnu[j]; q++) o += "    fwd *= cG" + I(r.reactsp[j]) + ";\n";
    if (r.reversible) {
      o += "    double rev = K;\n";
      const char *f = r.nusum > 0.0 ? "prefRuTinv" : "prefRuT";
      for (int q = 0; q < (int)std::fabs(r.nusum); q++) o += std::string("    rev *= ") + f + ";\n";
      for (int j = 0; j < r.nprod; j++)
        for (int q = 0; q < (int)r.prodnu[j]; q++) o += "    rev *= cG" + I(r.prodsp[j]) + ";\n";
    }
  } else {
    if (thirdbody && !falloff) o += "    lk += logtb" + I(r.tb) + ";\n";
    if (falloff) o += "    lk += fmin(logpr, 0.0) - log1p(texp(-fabs(logpr), mt));\n";
    if (r.kind == 3) troe(m, r, o);
    o += "    double lrp = lk;\n";
    for (int j = 0; j < r.nfwd; j++) o += "    lrp += " + lit(r.fwdorder[j]) + " * logc" + I(r.fwdsp[j]) + ";\n";
    o += "    const double fwd = texp(fmin(lrp, " + clamp + "), mt);\n";
    if (r.reversible) {
      o += "    double diff = " + (r.nusum != 0.0 ? lit(r.nusum) + " * logprefRuT" : std::string("0.0")) + ";\n";
      for (int j = 0; j < r.nnet; j++)
        o += "    diff -= " + lit(r.netnu[j]) + " * (gRT" + I(r.netsp[j]) + " + logc" + I(r.netsp[j]) + ");\n";
      o += "    const double rev = texp(fmin(lrp - diff, " + clamp + "), mt);\n";
    }
  }
  o += r.reversible ? "    const double rp = fwd - rev;\n" : "    const double rp = fwd;\n";
  for (int j = 0; j < r.nnet; j++) o += "    omega" + I(r.netsp[j]) + " += " + lit(r.netnuMW[j]) + " * rp;\n";
  o += "  }\n";
}

}  // namespace

std::string rates_source(const Mech &m, const Species &sp, int ns) {
  const int ne = 4 + ns;
  std::string o = kPrelude;
  o += "\nextern \"C\" __global__ void __launch_bounds__(256) pgb_gen_source(\n"
       "    const char *__restrict__ blks, const int stride, const int b, const double *__restrict__ Qall,\n"
       "    const double *__restrict__ stall, double *__restrict__ dQall, const TileRef *__restrict__ ctab,\n"
       "    const MathTables *__restrict__ mt) {\n";
  // the cell (layout.cuh: PGB_WHERE, cell_index; chem.cuh: k_source)
  o += "  const TileRef w = ctab ? ctab[blockIdx.x] : TileRef{b + (int)blockIdx.y, (int)blockIdx.x};\n"
       "  const BlockHead &B = *reinterpret_cast<const BlockHead *>(blks + (long long)w.x * stride);\n"
       "  const long long t = (long long)w.y * blockDim.x + threadIdx.x;\n"
       "  if (t >= (long long)B.nx * B.ny * B.nz) return;\n"
       "  const int i = (int)(t % B.nx) + " + I(NG) + ", j = (int)((t / B.nx) % B.ny) + " + I(NG) +
       ", k = (int)(t / ((long long)B.nx * B.ny)) + " + I(NG) + ";\n"
       "  const long long c = (long long)i + (long long)B.X * ((long long)j + (long long)B.Y * k), v = B.vol;\n"
       "  const double *Q = Qall + " + I(ne) + " * B.cv + c;\n"
       "  const double T = stall[" + I(SW) + " * B.cv + 1 * v + c];\n";
  // cellrates: the clipped mass fractions
  o += "  const double rho = Q[0], rhoinv = 1.0 / rho;\n  double Ylast = 1.0, Ysum = 0.0;\n";
  for (int n = 0; n < ns - 1; n++)
    o += "  {\n    const double Yn = fmax(fmin(Q[" + I(5 + n) + " * v] * rhoinv, 1.0), 0.0);\n"
         "    Ylast -= Yn;\n    Ysum += Yn;\n  }\n";
  o += "  const double Yscale = 1.0 / fmax(Ysum, 1.0);\n  Ylast = fmax(Ylast, 0.0);\n";
  // ratestate
  o += "  const double logT = tlog(T, mt);\n  const double Tinv = 1.0 / T;\n";
  o += "  const double logprefRuT = " + lit(m.logprefRu) + " - logT;\n";
  o += "  const double prefRuT = " + lit(m.prefRu) + " * Tinv;\n";
  o += "  const double prefRuTinv = " + lit(m.Rupref) + " * T;\n  double ctot = 0.0;\n";
  for (int n = 0; n < ns; n++) {
    const std::string N = I(n);
    if (n < ns - 1)
      o += "  const double Y" + N + " = fmax(fmin(Q[" + I(5 + n) + " * v] * rhoinv, 1.0), 0.0) * Yscale;\n";
    else
      o += "  const double Y" + N + " = Ylast;\n";
    o += "  const double c" + N + " = rho * Y" + N + " * " + lit(sp.MWinv[n]) + ";\n  ctot += c" + N + ";\n";
    o += "  double gRT" + N + ";\n  {\n    double g = 0.0;\n";
    for (int tt = MAXT; tt >= 0; tt--)
      if (tt < m.ngp) o += "    g = g * logT + " + lit(m.gpoly[n][tt]) + ";\n";
    o += "    gRT" + N + " = g + " + lit(sp.h298[n]) + " * Tinv;\n  }\n";
    if (m.logform) o += "  const double logc" + N + " = fmax(" + lit(m.logcfloor) + ", tlog(c" + N + ", mt));\n";
    if (m.product) o += "  const double cG" + N + " = fmax(c" + N + ", 0.0) * texp(gRT" + N + ", mt);\n";
  }
  for (int jt = 0; jt < m.ntb; jt++) {
    const std::string J = I(jt);
    o += "  double ctb" + J + " = " + lit(m.tbdefeff[jt]) + " * ctot;\n";
    for (int q = 0; q < m.tbneff[jt]; q++)
      o += "  ctb" + J + " += " + lit(m.tbeffdev[jt][q]) + " * (rho * Y" + I(m.tbeffsp[jt][q]) + " * " +
           lit(sp.MWinv[m.tbeffsp[jt][q]]) + ");\n";
    o += "  const double logtb" + J + " = tlog(fmax(2.2250738585072014e-308, ctb" + J + "), mt);\n";
  }
  // the fold
  for (int n = 0; n < ns; n++) o += "  double omega" + I(n) + " = 0.0;\n";
  for (int k = 0; k < m.nr; k++) reaction(m, m.rxn[k], k, o);
  // dQ begins with the source
  o += "  double *dQ = dQall + " + I(ne) + " * B.cv + c;\n";
  for (int l = 0; l < 5; l++) o += "  dQ[" + I(l) + " * v] = 0.0;\n";
  for (int n = 0; n < ns - 1; n++) o += "  dQ[" + I(5 + n) + " * v] = omega" + I(n) + ";\n";
  o += "}\n";
  return o;
}

namespace {

// NVRTC's entry points, opened at run time
struct Nvrtc {
  bool ok = false;
  std::string why;
  typedef int (*Create)(void **, const char *, const char *, int, const char *const *, const char *const *);
  typedef int (*Compile)(void *, int, const char *const *);
  typedef int (*Size)(void *, size_t *);
  typedef int (*Get)(void *, char *);
  typedef int (*Destroy)(void **);
  Create create = nullptr;
  Compile compile = nullptr;
  Size logsize = nullptr, cubinsize = nullptr;
  Get log = nullptr, cubin = nullptr;
  Destroy destroy = nullptr;
  Nvrtc() {
    const char *names[] = {"libnvrtc.so.12", "libnvrtc.so", "/usr/local/cuda/lib64/libnvrtc.so.12"};
    void *h = nullptr;
    for (const char *n : names)
      if ((h = dlopen(n, RTLD_NOW | RTLD_LOCAL))) break;
    if (!h) {
      why = "NVRTC (libnvrtc.so.12) could not be opened";
      return;
    }
    create = (Create)dlsym(h, "nvrtcCreateProgram");
    compile = (Compile)dlsym(h, "nvrtcCompileProgram");
    logsize = (Size)dlsym(h, "nvrtcGetProgramLogSize");
    log = (Get)dlsym(h, "nvrtcGetProgramLog");
    cubinsize = (Size)dlsym(h, "nvrtcGetCUBINSize");
    cubin = (Get)dlsym(h, "nvrtcGetCUBIN");
    destroy = (Destroy)dlsym(h, "nvrtcDestroyProgram");
    ok = create && compile && logsize && log && cubinsize && cubin && destroy;
    if (!ok) why = "NVRTC lacks an entry point this library calls";
  }
};

}  // namespace

bool rates_compile(const std::string &src, std::string &out, std::string &err) {
  static Nvrtc nv;
  if (!nv.ok) {
    err = nv.why;
    return false;
  }
  void *prog = nullptr;
  if (nv.create(&prog, src.c_str(), "pgb_gen_source.cu", 0, nullptr, nullptr) != 0) {
    err = "nvrtcCreateProgram failed";
    return false;
  }
  // the library's own device code is built -O3 with contraction on, no fast math
  const char *opts[] = {"--gpu-architecture=sm_100a", "-std=c++17", "--fmad=true"};
  const int rc = nv.compile(prog, 3, opts);
  size_t n = 0;
  nv.logsize(prog, &n);
  std::string log(n, '\0');
  if (n) nv.log(prog, &log[0]);
  if (rc != 0) {
    err = "the generated source did not compile:\n" + log;
    nv.destroy(&prog);
    return false;
  }
  nv.cubinsize(prog, &n);
  out.assign(n, '\0');
  nv.cubin(prog, &out[0]);
  nv.destroy(&prog);
  return true;
}

}  // namespace pgb
