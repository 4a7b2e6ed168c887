// Shared internals of libsbh_b200.so (not part of the C ABI).
#pragma once

#include <string>

#include "../../include/sbh_b200.h"
#include "host_tree.h"

#define SBH_API extern "C" __attribute__((visibility("default")))

struct sbh_host_tree {
  sbh::HostTree t;
};

namespace sbh {

// Records a thread-local error message and returns `status`.
int fail(int status, const std::string& msg);
// Clears the thread-local error message and returns SBH_OK.
int ok();
// Fills `info` from a host tree (device_bytes = 0).
void fill_info(const HostTree& t, sbh_tree_info* info);

}  // namespace sbh
