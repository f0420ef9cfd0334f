"""Write C stubs for symbols the reference oracle leaves undefined.

Test infrastructure only. The reference sources compiled by oracle/ref/Makefile pull in
file-I/O libraries that are absent here (libtiff, cfitsio, libxml2, NeXus/HDF5) and a
few kipl helpers that sit off the hot path. None of them is called on the paths the
harness drives (inputs are in-memory, configs are set in code), so each undefined
function gets a stub that aborts loudly if it is ever reached.

usage: python gen_stubs.py <undefined-symbols.txt> <out.c>
"""
import sys

IGNORE = {"__gmon_start__", "_ITM_deregisterTMCloneTable", "_ITM_registerTMCloneTable"}


def main() -> None:
    src, dst = sys.argv[1], sys.argv[2]
    names = []
    with open(src) as f:
        for line in f:
            name = line.strip()
            if not name or name in IGNORE or "@" in name:
                continue
            names.append(name)
    with open(dst, "w") as f:
        f.write("/* generated by oracle/ref/gen_stubs.py: off-path symbols of the reference oracle */\n")
        f.write("#include <stdio.h>\n#include <stdlib.h>\n")
        f.write("static void oracle_stub_hit(const char *n) { fprintf(stderr, \"reference oracle: off-path symbol %s called\\n\", n); abort(); }\n")
        for n in sorted(set(names)):
            f.write(f"void {n}(void) {{ oracle_stub_hit(\"{n}\"); }}\n")


if __name__ == "__main__":
    main()
