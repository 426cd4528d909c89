// Include-path overlay: pe's own pe/core/collisionsystem/Default.h, then the B200 collision
// system specialisations.  pe/core/CollisionSystem.h includes this file last among its
// specialisations, right before it names CollisionSystem<Config>, so the B200 specialisations
// are declared before pe's configuration instantiates the collision system.
#include_next <pe/core/collisionsystem/Default.h>
#include <pe_b200_pe/pe_b200_collision_system.h>
