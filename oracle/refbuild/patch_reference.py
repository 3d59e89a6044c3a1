#!/usr/bin/env python3
"""Copy the reference solver sources into a scratch build directory and apply
the small compile fixes GCC needs.

The reference was written for MSVC, which accepts some dead template code and
a few non-standard constructs that GCC rejects.  Every edit below is a compile
fix only (typos in code that is never instantiated on the solver path, open
modes, a glibc-unsafe vsprintf self-overlap, iterator/temporary binding); none
changes the arithmetic of the solver path.  The scratch copy lives under
oracle/_ref/ (git-ignored) and is deleted by the Makefile after the build.

Usage: patch_reference.py <reference_dir> <scratch_dir>
"""
import os
import shutil
import sys

# (file, original fragment, replacement).  Each fragment must occur exactly
# `count` times in the file, otherwise the recipe stops: the reference changed
# and the edit list has to be reviewed.
EDITS = [
    ("ARRAY_3D.h", "values[i] -= constant;", "values[i] -= costant;", 1),
    ("ARRAY_2D.h", "values[i] -= constant;", "values[i] -= costant;", 1),
    ("ARRAY_3D.h", "\t\tasset(", "\t\tassert(", 1),
    ("CSR_MATRIX.h", "value_ix = matrix_input.value_ix;", "values_ix = matrix_input.values_ix;", 1),
    ("CSR_MATRIX.h", "prev_row_array_[thread_id]", "prev_row_array[thread_id]", 1),
    ("CSR_MATRIX.h", "xval[column_index_[vix]]", "xval[column_index[vix]]", 1),
    ("FIELD_STRUCTURE_3D.h", "const TT& componentwise_max)\n\t{\n\t\tconst T &posx(pos.x), &posy(pos.y), &posz(pos.z);",
     "const TT& componentwise_max)\n\t{\n\t\tconst T &posx(position.x), &posy(position.y), &posz(position.z);", 1),
    ("FIELD_STRUCTURE_3D.h", "*(values + ((CLAMP(ix.i,i_start_g,i_end_g) - i_start_g) + (CLAMP(ix.j,j_start_g,j_end_g) - j_start_g)*i_res_g + (CLAMP(ix.k,k_start_g,k_end_g) - k_start_g)*ij_res_g",
     "*(values + ((CLAMP(i,i_start_g,i_end_g) - i_start_g) + (CLAMP(j,j_start_g,j_end_g) - j_start_g)*i_res_g + (CLAMP(k,k_start_g,k_end_g) - k_start_g)*ij_res_g", 1),
    ("FIELD_STRUCTURE_3D.h", "std::memset(array_for_this.values", "memset(array_for_this.values", 1),
    ("LOG.h", "ios_base::trunc || ios_base::out", "ios_base::trunc | ios_base::out", 3),
    ("LOG.h", "\t\t\tBegin(va_buffer);\n\t\t}\n\t\tEND_HEAD_THREAD_WORK",
     "\t\t\tstatic char va_copy_buffer[sizeof(va_buffer)]; memcpy(va_copy_buffer, va_buffer, sizeof(va_buffer)); Begin(\"%s\", va_copy_buffer);\n\t\t}\n\t\tEND_HEAD_THREAD_WORK", 1),
    ("RIGID_OBJECT.h", "rotation = MATRIX_3X3::Identity();",
     "{ MATRIX_3X3 identity_tmp = MATRIX_3X3::Identity(); rotation = identity_tmp; }", 2),
    ("SCRIPT_READER.cpp", "string(preprocessed_script.data(), matches[0].first)",
     "string((const char*)preprocessed_script.data(), (const char*)matches[0].first)", 1),
    ("SCRIPT_READER.cpp", "values.swap(vector<SCRIPT_VALUE*>());", "vector<SCRIPT_VALUE*>().swap(values);", 1),
    ("TRIANGULAR_SURFACE.cpp", "if(ist == NULL)", "if(ist.fail())", 1),
    ("TRIANGULAR_SURFACE.cpp", "if(file == 0)", "if(file.fail())", 1),
    # std::thread passes its arguments as rvalues, which GCC will not bind to
    # the int& thread ids of the polygonizer's thread functions (MSVC does)
    ("MARCHING_CUBES_ALGORITHM.h", "void PolygonizeThread(int& thread_id, LEVELSET_OBJECT* levelset)",
     "void PolygonizeThread(int thread_id, LEVELSET_OBJECT* levelset)", 1),
    ("MARCHING_CUBES_ALGORITHM.h", "void PolygonizeUseFillGhostCellsFromThread(int& thread_id, LEVELSET_3D* levelset)",
     "void PolygonizeUseFillGhostCellsFromThread(int thread_id, LEVELSET_3D* levelset)", 1),
    ("MARCHING_CUBES_ALGORITHM.h", "void PolygonizeThreadPeriodic(int& thread_id, LEVELSET_OBJECT* levelset",
     "void PolygonizeThreadPeriodic(int thread_id, LEVELSET_OBJECT* levelset", 1),
]


# The moving-least-squares class is off the solver path (it only seeds a level
# set from particles) and its matrix helpers do not compile under GCC; the
# level set only needs the type and one query, so a stub replaces the header.
MLS_STUB = """#pragma once
#include "COMMON_DEFINITIONS.h"
class MOVING_LEAST_SQUARES
{
public:
	T GetScalar(const VT&) const { return (T)0; }
};
"""


def main():
    ref, out = sys.argv[1], sys.argv[2]
    os.makedirs(out, exist_ok=True)
    for name in os.listdir(ref):
        if name.endswith((".h", ".cpp")):
            shutil.copyfile(os.path.join(ref, name), os.path.join(out, name))
    for fname, old, new, count in EDITS:
        path = os.path.join(out, fname)
        with open(path, encoding="latin-1") as f:
            text = f.read()
        found = text.count(old)
        if found != count:
            sys.exit(f"patch_reference: {fname}: expected {count} occurrence(s) of {old!r}, found {found}")
        with open(path, "w", encoding="latin-1") as f:
            f.write(text.replace(old, new))
    with open(os.path.join(out, "MOVING_LEAST_SQUARES.h"), "w") as f:
        f.write(MLS_STUB)
    print(f"patch_reference: {len(EDITS)} edits applied in {out}")


if __name__ == "__main__":
    main()
