// ProtoMol module registering the libpmgpu GPU forces with the force
// factory and the device-resident integrators with the integrator factory
// (the patterns of module/BondedForcesModule.h and module/LeapfrogModule.h).
#ifndef PMGPU_FORCE_MODULE_H
#define PMGPU_FORCE_MODULE_H

#include <protomol/base/Module.h>

#include <string>

namespace ProtoMol {
class ProtoMolApp;

class PmgpuForceModule : public Module {
 public:
  const std::string getName() const { return "PmgpuForces"; }
  int getPriority() const { return 0; }
  const std::string getHelp() const {
    return "GPU (B200) nonbonded cutoff, PME Ewald, GB, all-pairs and torsion forces; "
           "LeapfrogGPU and LangevinLeapfrogGPU device-resident integrators";
  }
  void registerForces(ProtoMolApp *app);

 protected:
  void init(ProtoMolApp *app);
};
}  // namespace ProtoMol

#endif
