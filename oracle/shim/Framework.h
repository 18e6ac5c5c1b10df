// Include shim for the oracle build: RLGymCPP's CommonValues.h includes "../Framework.h"
// relative to RLGymCPP/src, where no such file exists; the oracle build adds
// -I oracle/shim/inc so that this forwarder is found instead.
#pragma once
#include "RLGymCPP/Framework.h"
