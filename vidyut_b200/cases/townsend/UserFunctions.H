// The Townsend case uses the default transport and boundary callbacks
// (vidyut.user_defined_* = 0); it defines no user_transport hooks.
#pragma once
