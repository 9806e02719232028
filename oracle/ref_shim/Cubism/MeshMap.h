// Stand-in (oracle test infrastructure): the reference's uniform-grid path
// includes Cubism's mesh-map header but uses none of it.
#pragma once
