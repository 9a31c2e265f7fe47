#!/usr/bin/env python3
"""Emit the reference's generated limb<->point packers (test infrastructure).

The reference builds ``experiments/codegen/int_to_fft{b}.c`` and
``experiments/codegen/fft_to_int{b}.c`` (b = 7..22) with a Ruby generator
(experiments/codegen/gen.rb:83-235) that Ruby-less hosts cannot run.  This
module restates that generator's state machine so the reference sources
(fft/convert.c:8-40 #includes the outputs) can be compiled here as the CPU
oracle and baseline.  Nothing in the product imports it.

State machine (gen.rb:83-109 ``gencode``): walk one period of lcm(b, 32) bits
point by point; a point that stays inside one 32-bit word is one ``get`` and a
``put``; a point that straddles a word boundary takes the rest of the current
word, loads the next word (``ldf``, which may terminate the stream) and takes
the remaining low bits of that word.  The two emitters give the actions C code:

* int_to_fft (gen.rb:111-160): bit-slice the word stream into b-bit values,
  each written as the real part of one complex point (imaginary part 0).
* fft_to_int (gen.rb:162-208): scale the real part, round with
  ``(uint64_t)(f+0.5)``, add into a 64-bit carry and emit b bits at a time into
  32-bit words; the stream stops after exactly WL words.

Widths 2..6 (not generated by the reference, whose multiply aborts when it
would need them, bigfloat/mul.c:117-124 with fft/convert.c:66-68) can be
emitted with ``--widths 2-22`` for the extended oracle; they use the same
state machine.
"""
import argparse
import os


def _mask(bits):
    return "0x%x" % ((1 << bits) - 1)


def _walk(bpp):
    """Yield the generator's action list for one period (gen.rb:55-109)."""
    ops = [("init", bpp), ("ld",)]
    pos = 0
    while True:
        pw, pp = divmod(pos, 32)
        pos += bpp
        cw, cp = divmod(pos, 32)
        if pw == cw:
            ops.append(("get", cp - pp, cw, pp))
            ops.append(("put",))
        else:
            span = 32 * cw + cp - 32 * pw - pp
            ops.append(("get", 32 - pp, pw, pp))
            if cp % span != 0:
                ops.append(("ldf", cw))
                ops.append(("carry", cp))
                ops.append(("get", cp % span, cw, cp))
            ops.append(("put",))
        if cp == 0:
            break
    ops.append(("ret",))
    return ops


def emit_int_to_fft(bpp):
    out = []
    after_load = False
    last_bits = 0
    for op in _walk(bpp):
        kind = op[0]
        if kind == "init":
            out += [
                "// generated by oracle/gen_packers.py (restatement of experiments/codegen/gen.rb)",
                "static inline __attribute__((always_inline)) size_t int_to_fft%d(complex double *F, const uint32_t *W, size_t WL) {" % bpp,
                "  uint32_t w=0;",
                "  uint32_t c=0;",
                "  __m128d* T = (__m128d*)F;",
                "  const uint32_t *end = W + WL;",
                "  while(1) {",
            ]
        elif kind == "ld":
            out.append("    w = *W;")
        elif kind == "ldf":
            out += [
                "    if(++W >= end) {",
                "      *T++ = _mm_set_sd(c);",
                "      break;",
                "    }",
                "    w = *W;",
            ]
            after_load = True
        elif kind == "get":
            bits = op[1]
            if after_load:
                out.append("    c |= (w & %s) << %d;" % (_mask(bits), last_bits))
                after_load = False
            else:
                out.append("    c  |= w & %s;" % _mask(bits))
            out.append("    w >>= %d;" % bits)
            last_bits = bits
        elif kind == "put":
            out += ["    *T++ = _mm_set_sd(c);", "    c = 0;"]
        elif kind == "ret":
            out += [
                "    if(++W >= end) {",
                "      break;",
                "    }",
                "  }",
                "  return (complex double*)T - F;",
                "}",
                "",
            ]
    return "\n".join(out) + "\n"


def emit_fft_to_int(bpp):
    out = []
    after_load = False
    for op in _walk(bpp):
        kind = op[0]
        if kind == "init":
            out += [
                "// generated by oracle/gen_packers.py (restatement of experiments/codegen/gen.rb)",
                "static inline void fft_to_int%d(const complex double *F, uint32_t *W, size_t WL, double scale) {" % bpp,
                "  uint64_t c=0;",
                "  uint32_t *end = W + WL;",
                "  double f;",
                "  double i;",
                "  uint32_t w=0;",
                "  while(1) {",
            ]
        elif kind == "ldf":
            out += [
                "    *W = w;",
                "    if(++W >= end) {",
                "      break;",
                "    }",
                "    w = 0;",
            ]
            after_load = True
        elif kind == "get":
            bits, _word, bitpos = op[1], op[2], op[3]
            if after_load:
                out.append("    w |= c & %s;" % _mask(bits))
                out.append("    c >>= %d;" % bits)
                after_load = False
            else:
                out += [
                    "    f  = ((double*)F++)[0] * scale;",
                    "    i  = (uint64_t)(f+0.5);",
                    "    c += i;",
                    "    w |= (c&%s) << %d;" % (_mask(bits), bitpos),
                    "    c >>= %d;" % bits,
                ]
        elif kind == "ret":
            out += [
                "    *W = w;",
                "    if(++W >= end) {",
                "      break;",
                "    }",
                "    w = 0;",
                "  }",
                "}",
                "",
            ]
    return "\n".join(out) + "\n"


def _parse_widths(spec):
    lo, _, hi = spec.partition("-")
    return range(int(lo), int(hi or lo) + 1)


def main():
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--out", required=True, help="directory for the generated .c files")
    ap.add_argument("--widths", default="7-22", help="inclusive range, e.g. 7-22")
    args = ap.parse_args()
    os.makedirs(args.out, exist_ok=True)
    for b in _parse_widths(args.widths):
        for name, fn in (("int_to_fft", emit_int_to_fft), ("fft_to_int", emit_fft_to_int)):
            path = os.path.join(args.out, "%s%d.c" % (name, b))
            text = fn(b)
            old = None
            if os.path.exists(path):
                with open(path) as fh:
                    old = fh.read()
            if old != text:
                with open(path, "w") as fh:
                    fh.write(text)


if __name__ == "__main__":
    main()
