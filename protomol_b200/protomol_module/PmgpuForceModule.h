// ProtoMol module registering the libpmgpu GPU forces with the force
// factory (the pattern of module/BondedForcesModule.h).
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
    return "GPU (B200) nonbonded cutoff, PME Ewald and torsion forces";
  }
  void registerForces(ProtoMolApp *app);
};
}  // namespace ProtoMol

#endif
