// The LMEA case uses the default transport and boundary callbacks.
#pragma once
