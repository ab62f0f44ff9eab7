// Snapshot and checkpoint files (snapshot.cu) behind the handle's entry points.
#pragma once

#include <string>
#include <vector>

#include "../../include/treepm_b200.h"
#include "tree.cuh"

namespace tpm {

// The resident state a snapshot is written from: particles in storage order,
// the handle's box, a device staging buffer of at least 7 n doubles.
struct DeviceState {
  Particles p;
  int64_t n;
  double box;
  double* staging;
  cudaStream_t stream;
};

void snapshot_write(const std::string& dir, int32_t format, const tpm_snapshot_env* env, const tpm_provenance* prov,
                    const DeviceState& st);
void snapshot_write_host(const std::string& dir, int32_t format, const double* pos, const double* vel,
                         const double* mass, const uint64_t* ids, int64_t n, const tpm_snapshot_env* env,
                         const tpm_provenance* prov);
// Records in file order; env (may be null) from meta.json.
void snapshot_read(const std::string& dir, int32_t format, tpm_snapshot_env* env, std::vector<double>& pos,
                   std::vector<double>& vel, std::vector<double>& mass, std::vector<uint64_t>& ids);
// Reorder records into global-id order; the ids must be a permutation of 0..n-1.
void order_by_id(std::vector<double>& pos, std::vector<double>& vel, std::vector<double>& mass,
                 const std::vector<uint64_t>& ids);
void checkpoint_write_meta(const std::string& ck_dir, uint64_t completed_step, double a_current,
                           const char* config_hash, int64_t total);
void checkpoint_read_meta(const std::string& ck_dir, uint64_t* completed_step, double* a_current,
                          std::string* config_hash, int64_t* total);

}  // namespace tpm
