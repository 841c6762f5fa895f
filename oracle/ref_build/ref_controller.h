/* TEST INFRASTRUCTURE ONLY -- the pieces of the reference's CONTROLLER and
 * the global Xponge::system that its hot-path modules use, for the harnesses
 * that build those modules without control.cpp (which needs toml++) or the
 * Xponge loaders (which need HDF5).  Included by exactly one translation unit
 * of each harness library. */
#pragma once
#include <string>

#include "control.h"
#include "xponge/xponge.h"

/* ----------------------- CONTROLLER pieces ------------------------ */
unsigned int CONTROLLER::device_optimized_block = 64;
unsigned int CONTROLLER::device_warp = 32;
unsigned int CONTROLLER::device_max_thread = 1024;
int CONTROLLER::force_replica_count = 1;
int CONTROLLER::MPI_rank = 0;
int CONTROLLER::MPI_size = 1;
int CONTROLLER::PP_MPI_size = 1;
int CONTROLLER::PM_MPI_size = 1;
int CONTROLLER::CC_MPI_size = 1;
int CONTROLLER::PP_MPI_rank = 0;
int CONTROLLER::PM_MPI_rank = 0;
int CONTROLLER::CC_MPI_rank = 0;
int CONTROLLER::CV_MPI_rank = 0;
MPI_Comm CONTROLLER::pp_comm;
MPI_Comm CONTROLLER::pm_comm;
D_MPI_Comm CONTROLLER::D_MPI_COMM_WORLD;
D_MPI_Comm CONTROLLER::d_pp_comm;
D_MPI_Comm CONTROLLER::d_pm_comm;

CONTROLLER controller;
namespace Xponge
{
System system;
}


static std::string key_of(const char* prefix, const char* key)
{
    if (prefix == NULL || prefix[0] == 0) return key;
    return std::string(prefix) + "_" + key;
}
bool CONTROLLER::Command_Exist(const char* key) { return commands.count(key); }
bool CONTROLLER::Command_Exist(const char* prefix, const char* key)
{
    return commands.count(key_of(prefix, key));
}
const char* CONTROLLER::Command(const char* key)
{
    return commands[key].c_str();
}
const char* CONTROLLER::Command(const char* prefix, const char* key)
{
    return commands[key_of(prefix, key)].c_str();
}
bool CONTROLLER::Command_Choice(const char* key, const char* value,
                                bool case_sensitive)
{
    return commands.count(key) && commands[key] == value;
}
bool CONTROLLER::Command_Choice(const char* prefix, const char* key,
                                const char* value, bool case_sensitive)
{
    return Command_Choice(key_of(prefix, key).c_str(), value, case_sensitive);
}
TIME_RECORDER* CONTROLLER::Get_Time_Recorder(const char* name)
{
    return &time_recorders[name];
}
