// Include-path overlay for the compiled reference (oracle build only): selects pe's linear
// spring-dashpot normal force law (ForceModel 'basic', pe/core/response/ForceModel.h) instead
// of the Hertz default, as the benchmark workloads specify.  pe/system/DEMConfig.h includes
// this file inside namespace pe::dem.
const ForceModel forceModel = basic;
