"""Writes host-compilable copies of the decode kernels for the CPU emulation
test: the include paths point back at the package, the launchers (which
use the <<<>>> syntax) are dropped, dynamic shared memory becomes a static
buffer, and small wrappers expose each kernel to the driver."""
import pathlib
import re
import sys

CSRC = pathlib.Path(__file__).resolve().parents[2] / "signinum_b200" / "csrc"

HT_WRAPPERS = """
namespace sgn {
void emu_tables() { build_decode_tables(g_ht_tables); }
void emu_vlc(const HtJob* jobs, uint32_t n, const uint8_t* arena, uint32_t* sym, bool outline) {
  if (outline) ht_vlc_kernel<true>(jobs, n, arena, sym, 32);
  else ht_vlc_kernel<false>(jobs, n, arena, sym, 32);
}
void emu_magsgn(const HtJob* jobs, uint32_t n, const uint8_t* arena, const uint32_t* sym, int32_t* coef,
                uint32_t* status, uint32_t ms_words, uint32_t max_w, uint32_t nsingle) {
  ht_magsgn_kernel<false>(jobs, n, arena, sym, coef, status, ms_words, max_w, nullptr, 0, nsingle);
}
void emu_refine(const HtJob* jobs, const uint32_t* list, uint32_t n, const uint8_t* arena, int32_t* coef,
                uint32_t* status) {
  ht_refine_kernel(jobs, list, n, arena, coef, status);
}
void emu_fused(const HtJob* jobs, uint32_t n, const uint8_t* arena, uint32_t* sym, int32_t* coef, uint32_t* status,
               uint32_t ms_words, uint32_t max_w, bool outline) {
  if (outline) ht_cleanup_fused_kernel<true>(jobs, n, arena, sym, coef, status, ms_words, max_w);
  else ht_cleanup_fused_kernel<false>(jobs, n, arena, sym, coef, status, ms_words, max_w);
}
}  // namespace sgn
"""

CLASSIC_WRAPPERS = """
namespace sgn {
void emu_classic(const ClassicJob* jobs, const ClassicSeg* segs, uint32_t n, const uint8_t* arena,
                 const uint8_t* gather, int32_t* coef, uint16_t* scratch, uint32_t slot, uint32_t* queue) {
  QeTable qt;
  for (int i = 0; i < 47; ++i)
    qt.e[i] = ebcot::kQe[i] | ((uint32_t)ebcot::kNmps[i] << 16) | ((uint32_t)ebcot::kNlps[i] << 23) |
              ((uint32_t)ebcot::kSwitch[i] << 30);
  classic_kernel(jobs, segs, n, arena, gather, coef, scratch, slot, queue, qt);
}
}  // namespace sgn
"""

IP_WRAPPERS = """
namespace sgn {
void emu_idwt(bool irr, const IdwtJob* jobs, uint32_t n, uint32_t units) {
  if (irr) idwt97_level_kernel<false>(jobs, n, units, nullptr);
  else idwt_level_kernel<false>(jobs, n, units, nullptr);
}
template <int F>
void emu_pack_fmt(bool irr, const PackJob* jobs, uint32_t n, uint32_t units) {
  if (irr) return pack97_kernel<F, false>(jobs, n, units, nullptr);
  constexpr int NC = (F == PACK_GRAY8 || F == PACK_GRAY16) ? 1 : 3;
  // The launch's variant: every job of these launches has the first one's.
  if (pack_variant(F, jobs[0].ncomp, jobs[0].bit_depth) & 1) pack_kernel<F, NC, false, false>(jobs, n, units, nullptr);
  else pack_kernel<F, NC, true, false>(jobs, n, units, nullptr);
}
void emu_pack(bool irr, int fmt, const PackJob* jobs, uint32_t n, uint32_t units) {
#define K(F) case F: emu_pack_fmt<F>(irr, jobs, n, units); break;
  switch (fmt) { K(PACK_GRAY8) K(PACK_RGB8) K(PACK_RGBA8) K(PACK_GRAY16) K(PACK_RGB16) }
#undef K
}
int emu_pack_warps(bool irr) { return irr ? kWarps97 : kIdwtWarps; }
}  // namespace sgn
"""


def strip_functions(src, names):
    out, i = [], 0
    # A template header line directly above a launcher goes with it.
    pat = re.compile(r"^(template <[^>\n]*>\n)?(cudaError_t|size_t) (%s)\(" % names, re.M)
    while True:
        m = pat.search(src, i)
        if not m:
            out.append(src[i:])
            return "".join(out)
        out.append(src[i:m.start()])
        j, depth = src.index("{", m.start()), 0
        while True:
            depth += {"{": 1, "}": -1}.get(src[j], 0)
            if depth == 0 and src[j] == "}":
                break
            j += 1
        i = j + 1


def main(out_dir):
    out = pathlib.Path(out_dir)
    inc = lambda name: '#include "%s"' % (CSRC / name)
    src = (CSRC / "kernels" / "ht_decode.cu").read_text()
    src = src.replace('#include "../device_plan.h"', inc("device_plan.h"))
    src = src.replace('#include "../ht_tables.h"', inc("ht_tables.h"))
    src = src.replace('#include "kernels.h"', '#include "cuda_shim.h"\nnamespace sgn { size_t '
                      'ht_magsgn_smem_bytes(uint32_t ms_words, uint32_t max_w, uint32_t warps = 8); }')
    src = src.replace("extern __shared__ __align__(16) uint8_t smem[];", "uint8_t* smem = g_dyn_smem;")
    src = strip_functions(src, r"launch_\w+|ht_kernels_init|ht_magsgn_occupancy|upload_ht_tables")
    (out / "ht_decode_emu.cpp").write_text(src + HT_WRAPPERS)
    src = (CSRC / "kernels" / "idwt_pack.cu").read_text()
    src = src.replace('#include "../device_plan.h"', inc("device_plan.h")).replace('#include "kernels.h"',
                                                                                   '#include "cuda_shim.h"')
    src = strip_functions(src, r"launch_\w+|idwt_pack_occupancy")
    (out / "idwt_pack_emu.cpp").write_text(src + IP_WRAPPERS)
    src = (CSRC / "kernels" / "classic_decode.cu").read_text()
    src = src.replace('#include "../device_plan.h"', inc("device_plan.h")).replace('#include "../ebcot.h"', inc("ebcot.h"))
    src = src.replace('#include "kernels.h"', '#include "cuda_shim.h"')
    src = strip_functions(src, r"launch_\w+")
    src = re.sub(r"^uint32_t classic_threads_per_cta\(\) \{[^}]*\}", "", src, flags=re.M)
    src = src[:src.index("uint32_t classic_ctas_per_sm()")] + "}  // namespace sgn\n"
    (out / "classic_emu.cpp").write_text(src + CLASSIC_WRAPPERS)


if __name__ == "__main__":
    main(sys.argv[1])
