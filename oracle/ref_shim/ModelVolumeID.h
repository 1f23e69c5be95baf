// The reference's Model.h includes "ModelVolumeID.h" while the file on disk is
// ModelVolumnID.h; this forwards to it.
#include "ModelVolumnID.h"
