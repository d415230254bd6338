// Pass-specialised group-pass kernels: source generation, NVRTC compilation
// and launch. See jit.hpp.
#include "jit.hpp"
#include "plan.hpp"

#include <cuda.h>
#include <dlfcn.h>
#include <nvrtc.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <sstream>
#include <thread>

namespace kate {

namespace {

constexpr int TB = KATE_TILE_BITS;

uint32_t swz(uint32_t i) { return i ^ (((i >> 3) ^ (i >> 6) ^ (i >> 9)) & 7u); }

// Physical offset of tile slot x (swizzled element index) when tile bit k
// sits at physical bit pos[k]. Linear over GF(2) in x.
uint64_t slot_phys(uint32_t x, const uint8_t* pos) {
    const uint32_t e = swz(x);
    uint64_t o = 0;
    for (int k = 0; k < TB; k++)
        if ((e >> k) & 1u) o |= 1ull << pos[k];
    return o;
}

std::string hex(uint64_t v) {
    char b[32];
    std::snprintf(b, sizeof b, "0x%llxull", (unsigned long long)v);
    return b;
}
std::string hex32(uint32_t v) {
    char b[16];
    std::snprintf(b, sizeof b, "0x%xu", v);
    return b;
}

// Thread-bit vector i of stage si's shared-memory base (the stage tables are
// linear in the thread index: stab[v] for the low and high four bits).
uint32_t tvec(const PassProg& P, int si, int i) {
    return i < 4 ? P.stab[si][1 << i] : P.stab[si][16 + (1 << (i - 4))];
}
bool stage_linear(const PassProg& P, int si) {
    if (P.stab[si][0] != 0 || P.stab[si][16] != 0) return false;
    for (int v = 0; v < 16; v++) {
        uint32_t lo = 0, hi = 0;
        for (int i = 0; i < 4; i++)
            if ((v >> i) & 1) lo ^= P.stab[si][1 << i], hi ^= P.stab[si][16 + (1 << i)];
        if (lo != P.stab[si][v] || hi != P.stab[si][16 + v]) return false;
    }
    return true;
}
// Register vector j of table part `part` (32: load, 36: store).
uint32_t rvec(const PassProg& P, int si, int part, int j) {
    uint32_t r = 0;
    for (int i = 0; i < 4; i++)
        if ((j >> i) & 1) r ^= P.stab[si][part + i];
    return r;
}

const char* kPreamble = R"(
typedef unsigned int u32;
typedef unsigned long long u64;
#define S2I 0.7071067811865475
#define S2 1.4142135623730951
static __device__ __forceinline__ double2 mk(double x, double y) { return make_double2(x, y); }
static __device__ __forceinline__ double2 cmul(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
static __device__ __forceinline__ double2 row2(double2 u0, double2 u1, double2 x, double2 y) {
    double2 r;
    r.x = u0.x * x.x;
    r.x = fma(-u0.y, x.y, r.x);
    r.x = fma(u1.x, y.x, r.x);
    r.x = fma(-u1.y, y.y, r.x);
    r.y = u0.x * x.y;
    r.y = fma(u0.y, x.x, r.y);
    r.y = fma(u1.x, y.y, r.y);
    r.y = fma(u1.y, y.x, r.y);
    return r;
}
static __device__ __forceinline__ double2 row4(double2 u0, double2 u1, double2 u2, double2 u3, double2 x0, double2 x1,
                                                double2 x2, double2 x3) {
    double2 r;
    r.x = u0.x * x0.x;
    r.x = fma(-u0.y, x0.y, r.x);
    r.x = fma(u1.x, x1.x, r.x);
    r.x = fma(-u1.y, x1.y, r.x);
    r.x = fma(u2.x, x2.x, r.x);
    r.x = fma(-u2.y, x2.y, r.x);
    r.x = fma(u3.x, x3.x, r.x);
    r.x = fma(-u3.y, x3.y, r.x);
    r.y = u0.x * x0.y;
    r.y = fma(u0.y, x0.x, r.y);
    r.y = fma(u1.x, x1.y, r.y);
    r.y = fma(u1.y, x1.x, r.y);
    r.y = fma(u2.x, x2.y, r.y);
    r.y = fma(u2.y, x2.x, r.y);
    r.y = fma(u3.x, x3.y, r.y);
    r.y = fma(u3.y, x3.x, r.y);
    return r;
}
static __device__ __forceinline__ double2 lds(u32 a) {
    double2 v;
    asm volatile("ld.shared.v2.f64 {%0, %1}, [%2];" : "=d"(v.x), "=d"(v.y) : "r"(a));
    return v;
}
static __device__ __forceinline__ void sts(u32 a, double2 v) {
    asm volatile("st.shared.v2.f64 [%0], {%1, %2};" ::"r"(a), "d"(v.x), "d"(v.y) : "memory");
}
)";

struct Gen {
    const PassProg& P;
    std::ostringstream o;
    uint8_t in[TB], out[TB];
    explicit Gen(const PassProg& p) : P(p) {
        for (int k = 0; k < TB; k++) in[k] = out[k] = P.tphys[k];
        for (int i = 0; i < TB; i++) out[P.outsrc[i]] = P.tphys[i];
    }
    std::string thr_expr(const char* ty, int si, bool phys, const uint8_t* pos) {
        std::string e = std::string("(") + ty + ")0";
        for (int i = 0; i < 8; i++) {
            const uint32_t v = tvec(P, si, i);
            const uint64_t w = phys ? slot_phys(v >> 4, pos) : v;
            if (w == 0) continue;
            e += " ^ ((t & " + hex32(1u << i) + ") ? (" + ty + ")" + (phys ? hex(w) : hex32((uint32_t)w)) + " : (" +
                 ty + ")0)";
        }
        return e;
    }
    std::string cond(uint8_t cthr, uint64_t ccos) {
        std::string c = "true";
        if (cthr) c += " && ((t & " + hex32(cthr) + ") == " + hex32(cthr) + ")";
        if (ccos) c += " && ((cb & " + hex(ccos) + ") == " + hex(ccos) + ")";
        return c;
    }
    // Pair loop of a one-bit op on register bit b.
    template <typename F>
    void pairs(int b, F body) {
        for (int j = 0; j < 16; j++) {
            if ((j >> b) & 1) continue;
            const int k = j | (1 << b);
            o << "    { const double2 x = a" << j << ", y = a" << k << "; ";
            body(j, k);
            o << "}\n";
        }
    }
    std::string m(int i) { return "M.m[" + std::to_string(i) + "]"; }
};

bool lanes_ok(const PassProg& P, int st, const uint8_t* pos) {
    if (st < 0) return false;
    uint64_t acc = 0;
    for (int b = 0; b < 4; b++) {
        const uint64_t d = slot_phys((uint32_t)(P.stab[st][1 << b] ^ P.stab[st][0]) >> 4, pos);
        if (d == 0 || (d & (d - 1)) != 0) return false;
        acc |= d;
    }
    return acc == 15;
}

}  // namespace

bool jit_pass_work(const PassProg& P, double* fp64, double* smem) {
    std::string why;
    if (jit_pass_source(P, &why).empty()) return false;
    int first = -1, last = -1, exchanges = 0;
    double f = 0.0;
    for (int k = 0; k < P.nops; k++) {
        const SOp& op = P.ops[k];
        if (op.kind == SOP_STAGE) {
            if (first >= 0) exchanges++;
            if (first < 0) first = op.idx;
            last = op.idx;
        }
        f += sop_fp64_per_amp(op);
    }
    Gen g(P);
    double b = 32.0 * exchanges;
    if (!lanes_ok(P, first, g.in)) b += 32.0;
    if (!lanes_ok(P, last, g.out)) b += 32.0;
    *fp64 = f;
    *smem = b;
    return true;
}

std::string jit_pass_source(const PassProg& P, std::string* why, int form, int occ) {
    const bool from_zero = form == 1, from_prod = form == 2;
    auto no = [&](const char* w) {
        if (why) *why = w;
        return std::string();
    };
    if (P.m != TB || P.ncb < 0 || P.ncb > 22) return no("tile shape");
    int first = -1, last = -1;
    bool wide = false;
    for (int k = 0; k < P.nops; k++) {
        const int kind = P.ops[k].kind;
        if (kind == SOP_SMEM) return no("shared-memory op");
        if (kind == SOP_STAGE) {
            if (first >= 0 && P.ops[k].src != 1) wide = true;
            if (first < 0) first = P.ops[k].idx;
            last = P.ops[k].idx;
        } else if (first < 0 && kind != SOP_XL && kind != SOP_XF) {
            return no("register op before the first stage");
        }
    }
    if (first < 0) return no("no stage");
    for (int s = 0; s < P.nstages; s++)
        if (!stage_linear(P, s)) return no("stage table not linear");
    Gen g(P);
    // okL / okS: the first (last) stage's lanes 0..15 address physical bits
    // 0..3, so it reads (writes) HBM directly in 256-byte runs; otherwise the
    // tile is copied in (out) through shared memory in such runs.
    const bool okL = lanes_ok(P, first, g.in), okS = lanes_ok(P, last, g.out);
    (void)wide;
    std::ostringstream& o = g.o;
    int wbo[TB];
    for (int i = 0; i < TB; i++) wbo[i] = i;
    {
        // First three of output tile bits 0..3 whose input bits have
        // distinct residues mod 3, when there are such.
        int pick[3] = {-1, -1, -1}, np = 0;
        for (int a = 0; a < 4 && np < 3; a++)
            for (int b = a + 1; b < 4 && np < 3; b++)
                for (int c = b + 1; c < 4 && np < 3; c++) {
                    const int ra = P.outsrc[a] % 3, rb = P.outsrc[b] % 3, rc = P.outsrc[c] % 3;
                    if (ra != rb && rb != rc && ra != rc) pick[0] = a, pick[1] = b, pick[2] = c, np = 3;
                }
        if (np == 3) {
            wbo[0] = pick[0], wbo[1] = pick[1], wbo[2] = pick[2];
            wbo[3] = 6 - pick[0] - pick[1] - pick[2];
        }
    }
    const int nm = std::max(1, (int)P.nmats);
    o << kPreamble;
    o << "struct __align__(16) Mats { double2 m[" << nm << "]; };\n";
    if (from_prod) o << "struct __align__(16) ProdTab { double2 v[2][" << KATE_MAX_QUBITS << "]; };\n";
    o << "extern \"C\" __global__ void __launch_bounds__(256, " << occ
      << ") kate_pass(double2* __restrict__ st, const __grid_constant__ Mats M"
      << (from_prod ? ", const __grid_constant__ ProdTab PI" : "") << ") {\n";
    o << "  extern __shared__ __align__(16) unsigned char smem[];\n";
    o << "  const u32 tb = (u32)__cvta_generic_to_shared(smem);\n";
    o << "  const u32 t = threadIdx.x;\n";
    std::vector<char> used(P.nstages, 0);
    for (int k = 0; k < P.nops; k++)
        if (P.ops[k].kind == SOP_STAGE) used[P.ops[k].idx] = 1;
    for (int s = 0; s < P.nstages; s++)
        if (used[s] && s != first) o << "  const u32 s0_" << s << " = " << g.thr_expr("u32", s, false, nullptr) << ";\n";
    o << "  const u32 s0_" << first << " = " << g.thr_expr("u32", first, false, nullptr) << ";\n";
    if (okL) o << "  const u64 pin = " << g.thr_expr("u64", first, true, g.in) << ";\n";
    // Tile index (bit k = tile bit k, at physical bit tphys[k]) of a
    // physical offset made of tile bits only.
    auto tidx = [&](uint64_t x) {
        uint32_t r = 0;
        for (int k = 0; k < TB; k++)
            if ((x >> P.tphys[k]) & 1ull) r |= 1u << k;
        return r;
    };
    if (from_prod && okL) {
        std::string e = "(u32)0";
        for (int i = 0; i < 8; i++) {
            const uint32_t w = tidx(slot_phys(tvec(P, first, i) >> 4, g.in));
            if (w) e += " ^ ((t & " + hex32(1u << i) + ") ? " + hex32(w) + " : 0u)";
        }
        o << "  const u32 tin = " << e << ";\n";
    }
    if (okS) o << "  const u64 pout = " << g.thr_expr("u64", last, true, g.out) << ";\n";
    if (!okL || !okS) {
        // Copy j of thread t moves tile element t + 256 j: global offset
        // dT(t) ^ goff(j), shared offset swz(t + 256 j) << 4; on write-back
        // output element t + 256 j reads input slot pT(t) ^ osw(j).
        // The write-back's thread bits take the output tile bits in the
        // order wbo: bits 0..3 stay on lanes 0..3 (256-byte runs), with the
        // first three chosen so that the input slots they read lie in
        // distinct bank groups (tile bits of distinct residue mod 3 under
        // the swizzle), which keeps its shared-memory loads conflict-free.
        std::string dT = "(u64)0", dO = "(u64)0", sw = "(u32)0", pT = "(u32)0";
        for (int i = 0; i < 8; i++) {
            dT += " ^ ((t & " + hex32(1u << i) + ") ? (u64)" + hex(1ull << P.tphys[i]) + " : (u64)0)";
            dO += " ^ ((t & " + hex32(1u << i) + ") ? (u64)" + hex(1ull << P.tphys[wbo[i]]) + " : (u64)0)";
            sw += " ^ ((t & " + hex32(1u << i) + ") ? (u32)" + hex32(swz(1u << i) << 4) + " : (u32)0)";
            pT += " ^ ((t & " + hex32(1u << i) + ") ? (u32)" + hex32(swz(1u << P.outsrc[wbo[i]]) << 4) + " : (u32)0)";
        }
        o << "  const u64 cdT = " << dT << ";\n";
        if (!okL) o << "  const u32 csw = " << sw << ";\n";
        if (!okS) o << "  const u64 cdO = " << dO << ";\n  const u32 cpT = " << pT << ";\n";
    }
    // Coset index -> physical offset: runs of consecutive coset bits.
    // One coset per CTA: with no loop there is nothing loop-invariant for
    // the compiler to hoist into registers (the matrices stay constant-bank
    // operands instead of occupying registers across cosets).
    o << "  {\n    const u32 c = blockIdx.x;\n";
    o << "    u64 cb = 0;\n";
    for (int i = 0; i < P.ncb;) {
        int j = i;
        while (j + 1 < P.ncb && P.cphys[j + 1] == P.cphys[j] + 1) j++;
        const int len = j - i + 1;
        o << "    cb |= (u64)((c >> " << i << ") & " << hex32((uint32_t)((1ull << len) - 1)) << ") << " << (int)P.cphys[i]
          << ";\n";
        i = j + 1;
    }
    if (from_zero) {
        // The input is |0...0>: every coset but 0 is zero in and out, so its
        // output is written without being read or computed.
        o << "    if (c != 0) {\n      const double2 z = mk(0.0, 0.0);\n";
        if (okS) {
            o << "      const u64 b = cb ^ pout;\n";
            for (int j = 0; j < 16; j++)
                o << "      st[b ^ " << hex(slot_phys(rvec(P, last, 36, j) >> 4, g.out)) << "] = z;\n";
        } else {
            o << "      const u64 gb = cb ^ cdT;\n";
            for (int j = 0; j < 16; j++) {
                uint64_t go = 0;
                for (int i = 0; i < 4; i++)
                    if ((j >> i) & 1) go |= 1ull << P.tphys[8 + i];
                o << "      st[gb ^ " << hex(go) << "] = z;\n";
            }
        }
        o << "      return;\n    }\n";
    }
    if (from_prod) {
        // The input is the product state prod_p v[bit p][p]: its amplitude
        // is the coset's factor (the coset bits, once per CTA) times the
        // tile factor, read from two 64-entry tables (tile bits 0..5 and
        // 6..11) that the CTA builds first.
        o << "    __shared__ double2 ptl[64], pth[64];\n";
        o << "    double2 fc = mk(1.0, 0.0);\n";
        for (int i = 0; i < P.ncb; i++)
            o << "    fc = cmul(fc, ((cb >> " << (int)P.cphys[i] << ") & 1ull) ? PI.v[1][" << (int)P.cphys[i]
              << "] : PI.v[0][" << (int)P.cphys[i] << "]);\n";
        o << "    if (t < 128) {\n      const u32 u = t & 63u;\n      double2 f = mk(1.0, 0.0);\n";
        o << "      if (t < 64) {\n";
        for (int k = 0; k < 6; k++)
            o << "        f = cmul(f, ((u >> " << k << ") & 1u) ? PI.v[1][" << (int)P.tphys[k] << "] : PI.v[0]["
              << (int)P.tphys[k] << "]);\n";
        o << "        ptl[u] = f;\n      } else {\n";
        for (int k = 0; k < 6; k++)
            o << "        f = cmul(f, ((u >> " << k << ") & 1u) ? PI.v[1][" << (int)P.tphys[6 + k] << "] : PI.v[0]["
              << (int)P.tphys[6 + k] << "]);\n";
        o << "        pth[u] = f;\n      }\n    }\n    __syncthreads();\n";
    }
    o << "    double2 a0, a1, a2, a3, a4, a5, a6, a7, a8, a9, a10, a11, a12, a13, a14, a15;\n";
    o << "    u32 lfl = 0, sfl = 0; u64 lflp = 0, sflp = 0;\n";
    if (from_prod) o << "    u32 lflt = 0;\n";
    bool open = false, started = false;
    int si = -1;
    for (int k = 0; k < P.nops; k++) {
        const SOp& op = P.ops[k];
        switch (op.kind) {
        case SOP_STAGE: {
            if (open) {
                for (int j = 0; j < 16; j++)
                    o << "    sts(tb + ((s0_" << si << " ^ sfl) ^ " << hex32(rvec(P, si, 36, j)) << "), a" << j << ");\n";
            }
            si = op.idx;
            if (!started && from_prod) {
                if (okL) {
                    o << "    { const u32 ti = tin ^ lflt;\n";
                    for (int j = 0; j < 16; j++) {
                        const uint32_t tc = tidx(slot_phys(rvec(P, si, 32, j) >> 4, g.in));
                        o << "      { const u32 e = ti ^ " << hex32(tc) << "; a" << j
                          << " = cmul(fc, cmul(ptl[e & 63u], pth[e >> 6])); }\n";
                    }
                    o << "    }\n";
                } else {
                    // Element t + 256 j goes where the copy-in would have put it.
                    for (int j = 0; j < 16; j++)
                        o << "    { const u32 e = t | " << hex32((uint32_t)j << 8)
                          << "; sts(tb + (csw ^ " << hex32(swz((uint32_t)j << 8) << 4)
                          << "), cmul(fc, cmul(ptl[e & 63u], pth[e >> 6]))); }\n";
                    o << "    __syncthreads();\n";
                    o << "    { const u32 sl = s0_" << si << " ^ lfl;\n";
                    for (int j = 0; j < 16; j++)
                        o << "      a" << j << " = lds(tb + (sl ^ " << hex32(rvec(P, si, 32, j)) << "));\n";
                    o << "    }\n";
                }
                started = true;
            } else if (!started && from_zero) {
                // Coset 0 of |0...0>: the amplitude at global index 0 is 1.
                if (okL) {
                    o << "    { const u64 b = pin ^ lflp;\n";
                    for (int j = 0; j < 16; j++)
                        o << "      a" << j << " = mk((b ^ " << hex(slot_phys(rvec(P, si, 32, j) >> 4, g.in))
                          << ") == 0 ? 1.0 : 0.0, 0.0);\n";
                } else {
                    o << "    { const u32 sl = s0_" << si << " ^ lfl;\n";
                    for (int j = 0; j < 16; j++)
                        o << "      a" << j << " = mk((sl ^ " << hex32(rvec(P, si, 32, j)) << ") == 0 ? 1.0 : 0.0, 0.0);\n";
                }
                o << "    }\n";
                started = true;
            } else if (!started && !okL) {
                o << "    { const u64 gb = cb ^ cdT;\n";
                for (int j = 0; j < 16; j++) {
                    uint64_t go = 0;
                    for (int i = 0; i < 4; i++)
                        if ((j >> i) & 1) go |= 1ull << P.tphys[8 + i];
                    o << "      asm volatile(\"cp.async.cg.shared.global [%0], [%1], 16;\" :: \"r\"(tb + (csw ^ "
                      << hex32(swz((uint32_t)j << 8) << 4) << ")), \"l\"(st + (gb ^ " << hex(go) << ")) : \"memory\");\n";
                }
                o << "      asm volatile(\"cp.async.commit_group;\\n\\tcp.async.wait_group 0;\" ::: \"memory\");\n";
                o << "    }\n    __syncthreads();\n";
                o << "    { const u32 sl = s0_" << si << " ^ lfl;\n";
                for (int j = 0; j < 16; j++)
                    o << "      a" << j << " = lds(tb + (sl ^ " << hex32(rvec(P, si, 32, j)) << "));\n";
                o << "    }\n";
                started = true;
            } else if (!started) {
                o << "    { const u64 b = cb ^ pin ^ lflp;\n";
                for (int j = 0; j < 16; j++)
                    o << "      a" << j << " = __ldcg(st + (b ^ " << hex(slot_phys(rvec(P, si, 32, j) >> 4, g.in))
                      << "));\n";
                o << "    }\n";
                started = true;
            } else {
                o << (op.src == 1 ? "    __syncwarp();\n" : "    __syncthreads();\n");
                o << "    { const u32 sl = s0_" << si << " ^ lfl;\n";
                for (int j = 0; j < 16; j++)
                    o << "      a" << j << " = lds(tb + (sl ^ " << hex32(rvec(P, si, 32, j)) << "));\n";
                o << "    }\n";
            }
            o << "    lfl = 0; lflp = 0; sfl = 0; sflp = 0;\n";
            open = true;
            break;
        }
        case SOP_XF:
            o << "    if (" << g.cond(op.cthr, op.ccos) << ") { sfl ^= " << hex32(op.idx)
              << "; sflp ^= " << hex(slot_phys((uint32_t)op.idx >> 4, g.out)) << "; }\n";
            break;
        case SOP_XL:
            o << "    if (" << g.cond(op.cthr, op.ccos) << ") { lfl ^= " << hex32(op.idx)
              << "; lflp ^= " << hex(slot_phys((uint32_t)op.idx >> 4, g.in)) << ";";
            if (from_prod && !started) o << " lflt ^= " << hex32(tidx(slot_phys((uint32_t)op.idx >> 4, g.in))) << ";";
            o << " }\n";
            break;
        case SOP_U: {
            const int i = op.idx;
            g.pairs(op.a, [&](int j, int kk) {
                o << "a" << j << " = row2(" << g.m(i) << ", " << g.m(i + 1) << ", x, y); a" << kk << " = row2("
                  << g.m(i + 2) << ", " << g.m(i + 3) << ", x, y); ";
            });
            break;
        }
        case SOP_UR: {
            const int i = op.idx;
            const std::string u00 = g.m(i) + ".x", u01 = g.m(i + 1) + ".x", u10 = g.m(i + 2) + ".x",
                              u11 = g.m(i + 3) + ".x";
            g.pairs(op.a, [&](int j, int kk) {
                o << "a" << j << " = mk(fma(" << u01 << ", y.x, " << u00 << " * x.x), fma(" << u01 << ", y.y, " << u00
                  << " * x.y)); a" << kk << " = mk(fma(" << u11 << ", y.x, " << u10 << " * x.x), fma(" << u11
                  << ", y.y, " << u10 << " * x.y)); ";
            });
            break;
        }
        case SOP_UX: {
            const int i = op.idx;
            const std::string u00 = g.m(i) + ".x", u01 = g.m(i + 1) + ".y", u10 = g.m(i + 2) + ".y",
                              u11 = g.m(i + 3) + ".x";
            g.pairs(op.a, [&](int j, int kk) {
                o << "a" << j << " = mk(fma(-" << u01 << ", y.y, " << u00 << " * x.x), fma(" << u01 << ", y.x, "
                  << u00 << " * x.y)); a" << kk << " = mk(fma(-" << u10 << ", x.y, " << u11 << " * y.x), fma(" << u10
                  << ", x.x, " << u11 << " * y.y)); ";
            });
            break;
        }
        case SOP_URA:
        case SOP_URB:
        case SOP_UXA:
        case SOP_UXB: {
            const std::string t0 = g.m(op.idx) + ".x", t1 = g.m(op.idx) + ".y";
            g.pairs(op.a, [&](int j, int kk) {
                const std::string aj = "a" + std::to_string(j), ak = "a" + std::to_string(kk);
                if (op.kind == SOP_URA)
                    o << aj << " = mk(fma(" << t0 << ", y.x, x.x), fma(" << t0 << ", y.y, x.y)); " << ak << " = mk(fma("
                      << t1 << ", x.x, y.x), fma(" << t1 << ", x.y, y.y)); ";
                else if (op.kind == SOP_URB)
                    o << aj << " = mk(fma(" << t0 << ", x.x, y.x), fma(" << t0 << ", x.y, y.y)); " << ak << " = mk(fma("
                      << t1 << ", y.x, -x.x), fma(" << t1 << ", y.y, -x.y)); ";
                else if (op.kind == SOP_UXA)
                    o << aj << " = mk(fma(-" << t0 << ", y.y, x.x), fma(" << t0 << ", y.x, x.y)); " << ak
                      << " = mk(fma(-" << t1 << ", x.y, y.x), fma(" << t1 << ", x.x, y.y)); ";
                else
                    o << aj << " = mk(fma(" << t0 << ", x.y, y.x), fma(-" << t0 << ", x.x, y.y)); " << ak << " = mk(fma("
                      << t1 << ", y.y, x.x), fma(-" << t1 << ", y.x, x.y)); ";
            });
            break;
        }
        case SOP_U2: {
            const int i = op.idx, A = 1 << op.a, B = 1 << op.src;
            for (int j = 0; j < 16; j++) {
                if ((j & A) || (j & B)) continue;
                const int r[4] = {j, j | A, j | B, j | A | B};
                o << "    { const double2 x0 = a" << r[0] << ", x1 = a" << r[1] << ", x2 = a" << r[2] << ", x3 = a"
                  << r[3] << ";\n";
                for (int row = 0; row < 4; row++)
                    o << "      a" << r[row] << " = row4(" << g.m(i + 4 * row) << ", " << g.m(i + 4 * row + 1) << ", "
                      << g.m(i + 4 * row + 2) << ", " << g.m(i + 4 * row + 3) << ", x0, x1, x2, x3);\n";
                o << "    }\n";
            }
            break;
        }
        case SOP_H:
            g.pairs(op.a, [&](int j, int kk) {
                o << "const double2 n0 = mk((x.x + y.x) * S2I, (x.y + y.y) * S2I); a" << j << " = n0; a" << kk
                  << " = mk(n0.x - y.x * S2, n0.y - y.y * S2); ";
            });
            break;
        case SOP_X: {
            const std::string go = g.cond(op.cthr, op.ccos);
            o << "    { const bool go = " << go << ";\n";
            if (op.cthr == 0) o << "    if (go) {\n";
            for (int j = 0; j < 16; j++) {
                if ((j >> op.a) & 1) continue;
                if (((uint32_t)j & op.creg) != op.creg) continue;
                const int kk = j | (1 << op.a);
                if (op.cthr == 0)
                    o << "      { const double2 x = a" << j << "; a" << j << " = a" << kk << "; a" << kk << " = x; }\n";
                else
                    o << "      { const double2 x = a" << j << ", y = a" << kk << "; a" << j
                      << " = mk(go ? y.x : x.x, go ? y.y : x.y); a" << kk << " = mk(go ? x.x : y.x, go ? x.y : y.y); }\n";
            }
            if (op.cthr == 0) o << "    }\n";
            o << "    }\n";
            break;
        }
        case SOP_PH: {
            o << "    if (" << g.cond(op.cthr, op.ccos) << ") {\n";
            for (int j = 0; j < 16; j++)
                if (((uint32_t)j & op.creg) == op.creg) o << "      a" << j << " = cmul(a" << j << ", " << g.m(op.idx) << ");\n";
            o << "    }\n";
            break;
        }
        case SOP_D1: {
            const std::string bit = op.src == SRC_THR ? "((t >> " + std::to_string(op.a) + ") & 1u)"
                                                      : "((cb >> " + std::to_string(op.a) + ") & 1ull)";
            o << "    { const double2 d = " << bit << " ? " << g.m(op.idx + 1) << " : " << g.m(op.idx) << ";\n";
            for (int j = 0; j < 16; j++) o << "      a" << j << " = cmul(a" << j << ", d);\n";
            o << "    }\n";
            break;
        }
        case SOP_DR:
            for (int j = 0; j < 16; j++) o << "    a" << j << " = cmul(a" << j << ", " << g.m(op.idx + j) << ");\n";
            break;
        default:
            return no("unknown op");
        }
    }
    if (okS) {
        o << "    { const u64 b = cb ^ pout ^ sflp;\n";
        for (int j = 0; j < 16; j++)
            o << "      st[b ^ " << hex(slot_phys(rvec(P, si, 36, j) >> 4, g.out)) << "] = a" << j << ";\n";
        o << "    }\n";
    } else {
        for (int j = 0; j < 16; j++)
            o << "    sts(tb + ((s0_" << si << " ^ sfl) ^ " << hex32(rvec(P, si, 36, j)) << "), a" << j << ");\n";
        o << "    __syncthreads();\n    { const u64 gb = cb ^ cdO;\n";
        for (int j = 0; j < 16; j++) {
            uint64_t go = 0;
            uint32_t os = 0;
            for (int i = 0; i < 4; i++)
                if ((j >> i) & 1) go |= 1ull << P.tphys[wbo[8 + i]], os |= 1u << P.outsrc[wbo[8 + i]];
            o << "      st[gb ^ " << hex(go) << "] = lds(tb + (cpT ^ " << hex32(swz(os) << 4) << "));\n";
        }
        o << "    }\n";
    }
    o << "  }\n}\n";
    return o.str();
}

namespace {

// NVRTC and the driver API are resolved at run time, so the library loads
// (and its CPU-side entry points work) on machines without a GPU driver.
struct Api {
    nvrtcResult (*create)(nvrtcProgram*, const char*, const char*, int, const char* const*, const char* const*);
    nvrtcResult (*compile)(nvrtcProgram, int, const char* const*);
    nvrtcResult (*log_size)(nvrtcProgram, size_t*);
    nvrtcResult (*log)(nvrtcProgram, char*);
    nvrtcResult (*cubin_size)(nvrtcProgram, size_t*);
    nvrtcResult (*cubin)(nvrtcProgram, char*);
    nvrtcResult (*destroy)(nvrtcProgram*);
    const char* (*errstr)(nvrtcResult);
    CUresult (*mod_load)(CUmodule*, const void*);
    CUresult (*get_fn)(CUfunction*, CUmodule, const char*);
    CUresult (*set_attr)(CUfunction, CUfunction_attribute, int);
    CUresult (*occupancy)(int*, CUfunction, int, size_t);
    CUresult (*get_attr)(int*, CUfunction_attribute, CUfunction);
    CUresult (*launch)(CUfunction, unsigned, unsigned, unsigned, unsigned, unsigned, unsigned, unsigned, CUstream,
                       void**, void**);
    std::string nvrtc_err, drv_err;
    bool nvrtc_ok = false, drv_ok = false;
};

template <typename F>
bool sym(void* h, const char* name, F* out) {
    *out = reinterpret_cast<F>(dlsym(h, name));
    return *out != nullptr;
}

Api& api() {
    static Api a;
    static std::once_flag once;
    std::call_once(once, [] {
        const char* names[] = {"libnvrtc.so.12", "libnvrtc.so", "/usr/local/cuda/lib64/libnvrtc.so.12"};
        void* h = nullptr;
        for (const char* n : names)
            if ((h = dlopen(n, RTLD_NOW | RTLD_LOCAL))) break;
        if (!h) {
            a.nvrtc_err = "libnvrtc.so.12 not found";
        } else {
            a.nvrtc_ok = sym(h, "nvrtcCreateProgram", &a.create) && sym(h, "nvrtcCompileProgram", &a.compile) &&
                         sym(h, "nvrtcGetProgramLogSize", &a.log_size) && sym(h, "nvrtcGetProgramLog", &a.log) &&
                         sym(h, "nvrtcGetCUBINSize", &a.cubin_size) && sym(h, "nvrtcGetCUBIN", &a.cubin) &&
                         sym(h, "nvrtcDestroyProgram", &a.destroy) && sym(h, "nvrtcGetErrorString", &a.errstr);
            if (!a.nvrtc_ok) a.nvrtc_err = "libnvrtc.so.12 lacks an entry point";
        }
        auto drv = [](const char* name, void** p) {
            cudaDriverEntryPointQueryResult q;
            return cudaGetDriverEntryPoint(name, p, cudaEnableDefault, &q) == cudaSuccess &&
                   q == cudaDriverEntryPointSuccess && *p != nullptr;
        };
        a.drv_ok = drv("cuModuleLoadData", (void**)&a.mod_load) && drv("cuModuleGetFunction", (void**)&a.get_fn) &&
                   drv("cuFuncSetAttribute", (void**)&a.set_attr) &&
                   drv("cuOccupancyMaxActiveBlocksPerMultiprocessor", (void**)&a.occupancy) &&
                   drv("cuFuncGetAttribute", (void**)&a.get_attr) &&
                   drv("cuLaunchKernel", (void**)&a.launch);
        if (!a.drv_ok) a.drv_err = "CUDA driver entry points unavailable";
    });
    return a;
}

struct Cache {
    std::mutex mu;
    std::map<std::string, std::vector<char>> cubins;            // by source
    std::map<std::pair<int, std::string>, CUfunction> fns;      // by device and source
    std::map<CUfunction, int> occ;                              // CTAs per SM
};
Cache& cache() {
    static Cache c;
    return c;
}

std::string nvrtc_compile(const std::string& src, std::vector<char>* cubin) {
    Api& A = api();
    if (!A.nvrtc_ok) return A.nvrtc_err;
    nvrtcProgram prog;
    if (A.create(&prog, src.c_str(), "kate_pass.cu", 0, nullptr, nullptr) != NVRTC_SUCCESS)
        return "nvrtcCreateProgram failed";
    const char* opts[] = {"--gpu-architecture=sm_100a", "-std=c++17", "-default-device", "--fmad=true", "-lineinfo"};
    const nvrtcResult r = A.compile(prog, 5, opts);
    std::string err;
    if (r != NVRTC_SUCCESS) {
        size_t n = 0;
        A.log_size(prog, &n);
        std::string log(n, '\0');
        A.log(prog, &log[0]);
        err = std::string("NVRTC: ") + A.errstr(r) + "\n" + log.substr(0, 2000);
    } else {
        size_t n = 0;
        A.cubin_size(prog, &n);
        cubin->resize(n);
        A.cubin(prog, cubin->data());
    }
    A.destroy(&prog);
    return err;
}

}  // namespace

std::string jit_compile(int device, const std::vector<std::string>& srcs, std::vector<void*>* fns) {
    Cache& C = cache();
    fns->assign(srcs.size(), nullptr);
    std::vector<std::string> todo;
    {
        std::lock_guard<std::mutex> lk(C.mu);
        for (const auto& s : srcs)
            if (!C.cubins.count(s) && std::find(todo.begin(), todo.end(), s) == todo.end()) todo.push_back(s);
    }
    if (!todo.empty()) {
        std::vector<std::vector<char>> bins(todo.size());
        std::vector<std::string> errs(todo.size());
        const unsigned hw = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
        std::vector<std::thread> th;
        std::mutex qmu;
        size_t next = 0;
        for (unsigned w = 0; w < std::min<size_t>(hw, todo.size()); w++)
            th.emplace_back([&]() {
                for (;;) {
                    size_t i;
                    {
                        std::lock_guard<std::mutex> lk(qmu);
                        if (next >= todo.size()) return;
                        i = next++;
                    }
                    errs[i] = nvrtc_compile(todo[i], &bins[i]);
                }
            });
        for (auto& x : th) x.join();
        for (size_t i = 0; i < todo.size(); i++)
            if (!errs[i].empty()) return errs[i];
        std::lock_guard<std::mutex> lk(C.mu);
        for (size_t i = 0; i < todo.size(); i++) C.cubins[todo[i]] = std::move(bins[i]);
    }
    if (cudaSetDevice(device) != cudaSuccess || cudaFree(nullptr) != cudaSuccess) return "no CUDA context";
    Api& A = api();
    if (!A.drv_ok) return A.drv_err;
    std::lock_guard<std::mutex> lk(C.mu);
    for (size_t i = 0; i < srcs.size(); i++) {
        const auto key = std::make_pair(device, srcs[i]);
        auto it = C.fns.find(key);
        if (it == C.fns.end()) {
            CUmodule mod;
            CUfunction fn;
            CUresult r = A.mod_load(&mod, C.cubins[srcs[i]].data());
            if (r != CUDA_SUCCESS) return "cuModuleLoadData failed (" + std::to_string((int)r) + ")";
            r = A.get_fn(&fn, mod, "kate_pass");
            if (r != CUDA_SUCCESS) return "cuModuleGetFunction failed";
            A.set_attr(fn, CU_FUNC_ATTRIBUTE_MAX_DYNAMIC_SHARED_SIZE_BYTES, 65536);
            int occ = 1;
            if (A.occupancy(&occ, fn, 256, 65536) != CUDA_SUCCESS || occ < 1) occ = 1;
            C.occ[fn] = occ;
            it = C.fns.emplace(key, fn).first;
        }
        (*fns)[i] = (void*)it->second;
    }
    return "";
}

std::string jit_pass_key(const PassProg& P, int form, int occ) {
    std::string k;
    auto put = [&](const void* p, size_t n) { k.append(static_cast<const char*>(p), n); };
    const int32_t head[7] = {P.m, P.ncb, P.nops, P.nmats, P.nstages, form, occ};
    put(head, sizeof head);
    put(P.tphys, sizeof P.tphys);
    put(P.outsrc, sizeof P.outsrc);
    put(P.cphys, sizeof P.cphys);
    const int nops = std::max(0, std::min((int)P.nops, KATE_MAX_SOPS));
    const int nst = std::max(0, std::min((int)P.nstages, KATE_MAX_STAGES));
    put(P.ops, sizeof(SOp) * (size_t)nops);
    put(P.stab, sizeof(P.stab[0]) * (size_t)nst);
    put(P.srb, sizeof(P.srb[0]) * (size_t)nst);
    put(P.stb, sizeof(P.stb[0]) * (size_t)nst);
    return k;
}

namespace {
struct KeyCache {
    std::mutex mu;
    std::map<std::pair<int, std::string>, void*> fns;
};
KeyCache& key_cache() {
    static KeyCache c;
    return c;
}
}  // namespace

void* jit_find(int device, const std::string& key) {
    KeyCache& C = key_cache();
    std::lock_guard<std::mutex> lk(C.mu);
    auto it = C.fns.find(std::make_pair(device, key));
    return it == C.fns.end() ? nullptr : it->second;
}

void jit_remember(int device, const std::string& key, void* fn) {
    KeyCache& C = key_cache();
    std::lock_guard<std::mutex> lk(C.mu);
    C.fns[std::make_pair(device, key)] = fn;
}

int jit_local_bytes(void* fn) {
    int v = 0;
    if (!api().drv_ok || api().get_attr(&v, CU_FUNC_ATTRIBUTE_LOCAL_SIZE_BYTES, (CUfunction)fn) != CUDA_SUCCESS) return -1;
    return v;
}

int jit_grid(int ncb, int device) {
    (void)device;
    return 1 << ncb;  // one coset per CTA
}

cudaError_t jit_launch_prod(void* fn, void* st, const PassProg& prog, const ProdTab& pt, int grid, cudaStream_t s) {
    double2 mats[KATE_MAX_MATS];
    const int nm = std::max(1, (int)prog.nmats);
    for (int i = 0; i < nm; i++) mats[i] = make_double2(i < prog.nmats ? prog.mats[i][0] : 0.0, i < prog.nmats ? prog.mats[i][1] : 0.0);
    ProdTab p = pt;
    void* args[] = {&st, mats, &p};
    const CUresult r = api().launch((CUfunction)fn, grid, 1, 1, 256, 1, 1, 65536, (CUstream)s, args, nullptr);
    return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorLaunchFailure;
}

cudaError_t jit_launch(void* fn, void* st, const PassProg& prog, int grid, cudaStream_t s) {
    double2 mats[KATE_MAX_MATS];
    const int nm = std::max(1, (int)prog.nmats);
    for (int i = 0; i < nm; i++) mats[i] = make_double2(i < prog.nmats ? prog.mats[i][0] : 0.0, i < prog.nmats ? prog.mats[i][1] : 0.0);
    void* args[] = {&st, mats};
    const CUresult r = api().launch((CUfunction)fn, grid, 1, 1, 256, 1, 1, 65536, (CUstream)s, args, nullptr);
    return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorLaunchFailure;
}

}  // namespace kate
