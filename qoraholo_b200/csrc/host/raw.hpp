// Pointer forms of the per-call functions of include/qoraholo/*.hpp, for callers that hold their
// data in their own buffers (the Python bindings on numpy arrays): the same validation, errors and
// results as the Array3 forms, without copying the inputs into owning arrays or zero-filling the
// outputs first. Each function is split into a check (validation, output shape) and a run that
// writes into caller memory of that shape. Not part of the installed headers.
#pragma once

#include <array>
#include <span>

#include "qoraholo/qoraholo.hpp"

namespace qoraholo::raw {

// The first hologram of a (count, ny, nx) stack.
Sideband find_sideband(const float* holograms, int count, int ny, int nx, float dc_exclusion);

struct FieldCall {
  std::array<float, 2> center;  // the sideband centre used (given or detected)
  int out = 0;                  // output side m
};
FieldCall extract_fields_check(const float* holograms, int count, int ny, int nx, const FieldOptions& options,
                               Backend backend);
void extract_fields_run(const float* holograms, int count, int n, const FieldOptions& options, const FieldCall& call,
                        cfloat* out);

void field_ratio_check(int count, int ny, int nx, int bcount, int bny, int bnx);
void field_ratio_run(const cfloat* sample, int count, int ny, int nx, const cfloat* background, int bcount,
                     cfloat* out);

void unwrap_check(int ny, int nx, Backend backend);
void unwrap_run(const float* wrapped, int count, int ny, int nx, float* out);

void rytov_check(int ny, int nx, Backend backend);
void rytov_run(const cfloat* ratio, int count, int ny, int nx, cfloat* out);

// Returns nz.
int reconstruct_check(int count, int ny, int nx, std::span<const Illumination> illuminations, const Geometry& geometry,
                      const OdtOptions& options);
// Returns the filled fraction.
double reconstruct_run(const cfloat* fields, int count, int n, std::span<const Illumination> illuminations,
                       const Geometry& geometry, const OdtOptions& options, float* out);

}  // namespace qoraholo::raw
