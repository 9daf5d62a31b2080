// Shim: the reference's SIMT hop includes this external header but uses nothing from it.
#pragma once
