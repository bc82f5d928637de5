// The solver workload uses the default transport and boundary callbacks.
#pragma once
