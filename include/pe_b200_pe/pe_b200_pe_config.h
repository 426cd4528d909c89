/*
 * pe_b200_pe_config.h -- configuration fragment that makes pe's own World run its time step on
 * a B200 through libpe_b200.
 *
 * pe picks its collision system at compile time from four policies (pe/core/Configuration.h:84-88:
 * coarse detector, fine detector, batch generator, collision response; pe/config/Collisions.h:36,
 * 51, 67, 90).  Every rigid-body, contact and configuration trait of pe depends only on the
 * response, while the collision system is specialised on the whole policy set.  This fragment
 * selects a coarse-detector policy of its own, pe::detection::coarse::B200Detection; together with
 * pe's DEM response or its hard-contact response, that selects the CollisionSystem
 * specialisations of pe_b200_collision_system.h, which run detection, contact response and
 * integration of the whole step on the GPU, while bodies, materials, traits and the World stay
 * pe's.
 *
 * How pe is built with it (oracle/ref/Makefile, targets b200_dem and b200_hcsits, does exactly
 * this for pe's unmodified sources):
 *   1. the header pe's CMake build generates (cmake/config.h.in) defines pe_CONSTRAINT_SOLVER as
 *      pe::response::DEMSolver or pe::response::HardContactSemiImplicitTimesteppingSolvers and
 *      then includes this file;
 *   2. include/pe_b200_pe/overlay and include/ come before pe's own directory on the include path
 *      (the overlay's pe/core/collisionsystem/Default.h includes pe's file of that name and then
 *      the specialisations, at the point where pe/core/CollisionSystem.h declares its own);
 *   3. the program links libpe_b200.so and the CUDA runtime.
 */
#ifndef PE_B200_PE_CONFIG_H
#define PE_B200_PE_CONFIG_H

namespace pe {
namespace detection {
namespace coarse {
// the coarse-detector policy of the B200 collision system (defined in pe_b200_collision_system.h)
template <typename C>
class B200Detection;
}  // namespace coarse
}  // namespace detection
}  // namespace pe

#define pe_COARSE_COLLISION_DETECTOR ::pe::detection::coarse::B200Detection

#endif
