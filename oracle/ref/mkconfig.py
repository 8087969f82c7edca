"""Writes the configuration headers the reference's C++ needs into
<out>/SAMRAI/: SAMRAI_config.h, generated from the reference's own template
(config/SAMRAI_config.h.cmake.in) the way its CMake configure step would for
a serial (no MPI), HDF5-free, RAJA-free build, and an empty FC.h.

    python mkconfig.py <reference root> <out include dir>

TEST INFRASTRUCTURE ONLY: part of the recipe that builds the reference into
oracle/_ref/, the checker for the oracle and the CUDA path.
"""
import os
import re
import sys

DEFINED = {"HAVE_CMATH", "HAVE_STDLIB_H", "HAVE_STRING_H", "HAVE_UNISTD_H", "HAVE_SYS_TYPES_H",
           "HAVE_SYS_STAT_H", "HAVE_STDINT_H", "HAVE_INTTYPES_H", "HAVE_MEMORY_H",
           "HAVE_STRINGS_H", "HAVE_MALLOC_H", "HAVE_SYS_TIMES_H", "LACKS_MPI",
           "ENABLE_SAMRAI_TIMERS", "DEBUG_CHECK_ASSERTIONS", "INCLUDE_DEPRECATED"}
VALUES = {"SAMRAI_VERSION_MAJOR": "4", "SAMRAI_VERSION_MINOR": "0",
          "SAMRAI_VERSION_PATCHLEVEL": "1", "SAMRAI_MAXIMUM_DIMENSION": "3"}


def main(ref, out):
    src = open(os.path.join(ref, "config", "SAMRAI_config.h.cmake.in")).read()
    lines = []
    for line in src.splitlines():
        m = re.match(r"#cmakedefine\s+(\w+)", line)
        if m:
            if m.group(1) in DEFINED:
                lines.append(f"#define {m.group(1)}")
            continue
        line = re.sub(r"@(\w+)@", lambda mm: VALUES[mm.group(1)], line)
        # Fortran name mangling: lower case with one trailing underscore
        line = line.replace("#define SAMRAI_F77_FUNC CMAKE_FORTRAN_GLOBAL",
                            "#define SAMRAI_F77_FUNC(name, NAME) name##_")
        line = line.replace("#define SAMRAI_F77_FUNC_ CMAKE_FORTRAN_GLOBAL_",
                            "#define SAMRAI_F77_FUNC_(name, NAME) name##_")
        lines.append(line)
    d = os.path.join(out, "SAMRAI")
    os.makedirs(d, exist_ok=True)
    with open(os.path.join(d, "SAMRAI_config.h"), "w") as fh:
        fh.write("\n".join(lines) + "\n")
    with open(os.path.join(d, "FC.h"), "w") as fh:
        fh.write("/* no Fortran compiler configuration: names are mangled as name_ */\n")


if __name__ == "__main__":
    main(sys.argv[1], sys.argv[2])
