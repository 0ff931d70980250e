/* Oracle shim: archives are not used on the hot path. */
#pragma once
