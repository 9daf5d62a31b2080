// Shim for the reference's external qcu_io header qcu_helper.h (see qcu_public.h).
#pragma once
#include "qcu_public.h"
