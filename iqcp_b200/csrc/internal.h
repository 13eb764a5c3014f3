// Context accessors shared by the library's translation units (not part of
// the C ABI): host.cu owns struct iqcp_ctx, scf.cu drives the batched SCF
// through these and the public entry points.
#pragma once
#include <cuda_runtime.h>

#include <vector>

#include "engine.cuh"

struct iqcp_ctx;

namespace iqcp {
cudaStream_t ctx_stream(const iqcp_ctx* c);
int ctx_fail(iqcp_ctx* c, int code, const char* msg);
int ctx_device(const iqcp_ctx* c);
int ctx_n_mol(const iqcp_ctx* c);
const Packing& ctx_packing(const iqcp_ctx* c);            // device offsets of the packed matrices
const std::vector<long long>& ctx_mol_base(const iqcp_ctx* c);  // host: n_mol + 1 offsets
const std::vector<int>& ctx_mol_nbf(const iqcp_ctx* c);
const std::vector<int>& ctx_mol_atom0(const iqcp_ctx* c);       // n_mol + 1
const std::vector<int>& ctx_atom_z(const iqcp_ctx* c);
const std::vector<double>& ctx_atom_xyz(const iqcp_ctx* c);     // 3 per atom, bohr
// J/K and Fock builds skip the molecules whose flag is 0 (null: none skipped)
void ctx_set_mol_active(iqcp_ctx* c, const int* d_flags);
}  // namespace iqcp
