#include "../fenk.h"
