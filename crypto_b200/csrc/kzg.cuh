// KZG commit building blocks on device: fixed-base G1 multiplication (used
// to build synthetic SRS tables [tau^i]G1 and seeded input points s_i*G1),
// powers of tau in Fr, and the commit composition iNTT -> MSM -> compress.
#pragma once
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <string>

namespace kb200 {

class FixedBase;
FixedBase* fixed_base_create(int curve, cudaStream_t stream);  // builds the G table
void fixed_base_destroy(FixedBase* fb);
// out (table layout, 2N words per point, Montgomery affine) = s_i * G for
// n scalars (32-byte little-endian).  If out_wire is non-null the canonical
// big-endian wire encoding is written there as well.
void fixed_base_mul(FixedBase* fb, const uint8_t* d_scalars, size_t n, uint32_t* d_table_out,
                    uint8_t* d_wire_out, cudaStream_t stream);

// Shifted fixed-base tables over one resident BLS12-381 point table (an SRS
// or a blob setup): for window size c, msm_windows_for(c) levels of n rows,
// level w row i = [2^(c w)] (row i), built on first use and kept until the
// base changes.  Used with MsmOptions::shift_c / shift_stride.  Thread-safe.
struct ShiftTables;
ShiftTables* shift_tables_create();
void shift_tables_destroy(ShiftTables* t);
// New base table (device, n rows); drops every built level.
void shift_tables_reset(ShiftTables* t, const uint32_t* d_base, size_t n);
// Bumped by every reset (cache keys for anything holding level pointers).
uint64_t shift_tables_generation(const ShiftTables* t);
size_t shift_tables_stride(const ShiftTables* t);
// Levels for window size c (built and synchronised on `st` if new), or null
// when no base is set or the table would exceed its memory cap.
const uint32_t* shift_tables_get(ShiftTables* t, int c, cudaStream_t st);
// Window size minimising the modelled work of MSMs of these sizes against a
// shifted table.
int shift_c_for(const size_t* sizes, size_t count);
// Autotuner: shifted-table window (13, 16 or 19; 0 = cost model) of a
// single commit of 2^log_n evaluations.
void commit_tune_set(int log_n, int c);
int commit_tune_get(int log_n);
// Times single commits against the resident SRS per window (capi.cu).
int tune_commit_windows(int log_lo, int log_hi, const std::string& key, std::string& log);

// out[i] = tau^i (canonical 32-byte little-endian Fr), i < n.
void fr_powers(int curve, const uint8_t* d_tau, size_t n, uint8_t* d_out, cudaStream_t stream);

}  // namespace kb200
