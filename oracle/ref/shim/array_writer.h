// Headless stand-in for the reference's src/utils/array_writer.h, used only when the
// reference solver is compiled from source into oracle/_ref/ (test infrastructure).
//
// The reference header also pulls in libpng for image dumps; neither libpng nor any
// graphics stack exists on the build or GPU machines, so this stand-in provides only
// the text writers that src/algorithm/pppm.cu:4 needs (PPPMSolver::export_dirichlet,
// pppm.cu:416-421).  Output format: one "%e" value per line, no trailing newline, the
// format the reference documents for result.txt.
#pragma once
#include <cstdio>
#include <string>
#include "array3D.h"

namespace pppm
{

static inline void write_to_txt(std::string filename, const float *values, int count)
{
    FILE *out = fopen(filename.c_str(), "w");
    if (out == nullptr)
        return;
    for (int i = 0; i < count; i++)
        fprintf(out, i + 1 < count ? "%e\n" : "%e", values[i]);
    fclose(out);
}

template <typename T>
static inline void write_to_txt(std::string filename, CArr<T> values)
{
    write_to_txt(filename, values.data(), values.size());
}

}  // namespace pppm
