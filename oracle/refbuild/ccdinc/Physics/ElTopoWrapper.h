/* Empty stand-in for the El Topo wrapper header that Physics/SelfCollisionDetector.cpp
   includes but the reference does not ship; USE_EL_TOPO is off there, so nothing
   from it is used. Test infrastructure only. */
#pragma once
