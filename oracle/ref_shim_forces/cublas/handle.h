/* Host shim: the force code includes this header for a handle it does not use here. */
#pragma once
