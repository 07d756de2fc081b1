#!/usr/bin/env python3
"""Generate ``dvbt2_tables.h`` (the DVB-T2 LDPC parity-bit address tables).

The tables are the standard data of ETSI EN 302 755 V1.4.1 (Annex A for
normal frames, Annex B for short frames): for every 360-bit information
column block, the list of parity-check addresses ``x`` such that info bit
``block*360 + j`` participates in check ``(x + j*q) mod m``.

The erankavija/gf2 project (MIT licence) ships the same standard tables in
``crates/gf2-coding/src/ldpc/dvb_t2/dvb_t2_matrices.rs``; this script reads the
numbers out of that file once and writes them as compact C arrays.  The
generated header is committed, so building the library never needs the
source file.  Usage::

    python gen_dvbt2_tables.py /path/to/dvb_t2_matrices.rs > dvbt2_tables.h
"""
import re
import sys

# (frame, rate) -> (n, k, q) as given by DvbParams::for_code
# (crates/gf2-coding/src/ldpc/dvb_t2/params.rs:56-85).
PARAMS = {
    ("NORMAL", "1_2"): (64800, 32400, 90),
    ("NORMAL", "3_5"): (64800, 38880, 72),
    ("NORMAL", "2_3"): (64800, 43200, 60),
    ("NORMAL", "3_4"): (64800, 48600, 45),
    ("NORMAL", "4_5"): (64800, 51840, 36),
    ("NORMAL", "5_6"): (64800, 54000, 30),
    ("SHORT", "1_2"): (16200, 7200, 25),
    ("SHORT", "3_5"): (16200, 9720, 18),
    ("SHORT", "2_3"): (16200, 10800, 15),
    ("SHORT", "3_4"): (16200, 11880, 12),
    ("SHORT", "4_5"): (16200, 12600, 10),
    ("SHORT", "5_6"): (16200, 13320, 8),
}
RATES = ["1_2", "3_5", "2_3", "3_4", "4_5", "5_6"]


def parse(text):
    tables = {}
    for m in re.finditer(r"pub const (NORMAL|SHORT)_RATE_(\d_\d)_TABLE[^=]*=\s*&\[(.*?)\n\];",
                         text, re.S):
        frame, rate, body = m.group(1), m.group(2), m.group(3)
        rows = [[int(x) for x in r.split(",") if x.strip()]
                for r in re.findall(r"&\[([^\]]*)\]", body)]
        tables[(frame, rate)] = rows
    return tables


def main():
    src = open(sys.argv[1]).read()
    tables = parse(src)
    out = []
    out.append("// Generated by gen_dvbt2_tables.py -- do not edit.")
    out.append("// DVB-T2 LDPC parity-bit address tables, ETSI EN 302 755 V1.4.1 Annexes A/B")
    out.append("// (standard data; numbers as carried by erankavija/gf2, MIT licence).")
    out.append("#pragma once")
    out.append("#include <stdint.h>")
    out.append("")
    out.append("typedef struct {")
    out.append("  int n, k, q;            /* code length, info bits, address step */")
    out.append("  int rows;               /* info column blocks = k / 360 */")
    out.append("  const uint16_t* row_ptr; /* rows+1 offsets into addr */")
    out.append("  const uint16_t* addr;    /* parity-check base addresses */")
    out.append("} gf2_dvbt2_table_t;")
    out.append("")
    for frame in ("NORMAL", "SHORT"):
        for rate in RATES:
            rows = tables[(frame, rate)]
            n, k, q = PARAMS[(frame, rate)]
            assert len(rows) == k // 360, (frame, rate, len(rows))
            m = n - k
            assert all(0 <= x < m for r in rows for x in r)
            ptr = [0]
            flat = []
            for r in rows:
                flat.extend(r)
                ptr.append(len(flat))
            name = f"{frame.lower()}_{rate}"
            out.append(f"static const uint16_t gf2_dvbt2_{name}_ptr[{len(ptr)}] = {{")
            out.append(",".join(str(x) for x in ptr) + "};")
            out.append(f"static const uint16_t gf2_dvbt2_{name}_addr[{len(flat)}] = {{")
            for i in range(0, len(flat), 16):
                out.append(",".join(str(x) for x in flat[i:i + 16]) + ",")
            out.append("};")
    out.append("")
    out.append("/* index = frame * 6 + rate; frame 0 = normal (64800), 1 = short (16200);")
    out.append("   rate 0..5 = 1/2, 3/5, 2/3, 3/4, 4/5, 5/6 */")
    out.append("static const gf2_dvbt2_table_t gf2_dvbt2_tables[12] = {")
    for frame in ("NORMAL", "SHORT"):
        for rate in RATES:
            n, k, q = PARAMS[(frame, rate)]
            name = f"{frame.lower()}_{rate}"
            out.append(f"  {{{n}, {k}, {q}, {k // 360}, gf2_dvbt2_{name}_ptr, gf2_dvbt2_{name}_addr}},")
    out.append("};")
    print("\n".join(out))


if __name__ == "__main__":
    main()
