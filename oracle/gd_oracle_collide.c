/* placeholder translation unit, filled by the collision-operator restatement */
#include "gd_oracle.h"
