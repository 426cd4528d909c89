// Include-path overlay for the compiled reference (oracle build only): pe's extended Hertz
// normal force law for sphere-sphere contacts (ForceModel 'hertz', pe/core/response/ForceModel.h;
// pe's own default).  pe/system/DEMConfig.h includes this file inside namespace pe::dem.
const ForceModel forceModel = hertz;
